// Viscous stress divergence V_a = (1/Re) sum_b d/dx_b [mu (du_a/dx_b + du_b/dx_a)] / rho
// (ViscousSpatialEvaluator, src/twophase/ns_terms/viscous_spatial.py:28-153).
// The CCD first derivatives come from the CCD line kernels; this file holds
// the three-point low-order derivative of the stress (with the stress formed
// on the fly from mu and the two derivatives), the accumulation over b and
// the final division by Re rho.  Explicit round-to-nearest operations in the
// reference's NumPy order.
#include "tpf_common.cuh"

#include <algorithm>

namespace {

__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }

inline int blocks_for(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)tpf::sm_count() * 16));
}

struct LowArgs {
  const void *a, *b, *mu;         // value = mu (a + b), or a when mu is NULL (b NULL: a alone)
  const double *cl, *cc, *cr;     // interior coefficients per node along the axis (index k-1)
  double dx0, dxl;                // first and last cell widths
  void* total;
  const void* rho;
  double re;
  int64_t outer, n, inner;
  int accumulate, finalize;
};

template <typename T>
__device__ __forceinline__ double val(const LowArgs& a, int64_t i) {
  const double x = (double)static_cast<const T*>(a.a)[i];
  if (!a.mu) return x;
  const double y = a.b ? (double)static_cast<const T*>(a.b)[i] : 0.0;
  return rn_mul((double)static_cast<const T*>(a.mu)[i], a.b ? rn_add(x, y) : x);
}

// _low_order_derivative (viscous_spatial.py:70-104): one-sided first
// differences / dx at the ends, the three-point non-uniform stencil inside;
// then total (+)= it and, on the last axis, total / (Re rho).
template <typename T>
__global__ void lowfd_kernel(LowArgs a) {
  const int64_t tot = a.outer * a.n * a.inner;
  const int64_t s = a.inner, n = a.n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = (i / s) % n;
    double d;
    if (k == 0) {
      d = rn_sub(val<T>(a, i + s), val<T>(a, i)) / a.dx0;
    } else if (k == n - 1) {
      d = rn_sub(val<T>(a, i), val<T>(a, i - s)) / a.dxl;
    } else {
      const double fl = val<T>(a, i - s), fc = val<T>(a, i), fr = val<T>(a, i + s);
      d = rn_add(rn_add(rn_mul(a.cl[k - 1], fl), rn_mul(a.cc[k - 1], fc)), rn_mul(a.cr[k - 1], fr));
    }
    T* tot_p = static_cast<T*>(a.total);
    double t = a.accumulate ? rn_add((double)tot_p[i], d) : rn_add(0.0, d);
    if (a.finalize) t = t / rn_mul(a.re, (double)static_cast<const T*>(a.rho)[i]);
    tot_p[i] = (T)t;
  }
}

// stress = mu (a + b)  (the CCD-differentiated stress of the legacy scheme)
template <typename T>
__global__ void stress_kernel(int64_t n, const T* mu, const T* a, const T* b, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (T)rn_mul((double)mu[i], rn_add((double)a[i], (double)b[i]));
}

// total (+)= g, then (finalize) total / (Re rho)
template <typename T>
__global__ void accumulate_kernel(int64_t n, const T* g, int accumulate, int finalize, const T* rho, double re,
                                  T* total) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double t = accumulate ? rn_add((double)total[i], (double)g[i]) : rn_add(0.0, (double)g[i]);
    if (finalize) t = t / rn_mul(re, (double)rho[i]);
    total[i] = (T)t;
  }
}

}  // namespace

extern "C" int tpf_visc_lowfd_axis(int ndim, const int64_t* shape, int axis, const double* cl, const double* cc,
                                   const double* cr, double dx0, double dxl, const void* a, const void* b,
                                   const void* mu, int accumulate, int finalize, const void* rho, double re,
                                   void* total, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape && axis >= 0 && axis < ndim, "invalid shape or axis");
  TPF_CHECK_ARG(a && total && cl && cc && cr, "NULL argument");
  TPF_CHECK_ARG(total != a && total != b && total != mu, "total must not alias an operand");
  TPF_CHECK_ARG(!b || mu, "b is only used inside mu (a + b)");
  TPF_CHECK_ARG(!finalize || (rho && re != 0.0), "finalize needs rho and a nonzero Re");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  LowArgs A{};
  A.a = a; A.b = b; A.mu = mu; A.cl = cl; A.cc = cc; A.cr = cr; A.dx0 = dx0; A.dxl = dxl;
  A.total = total; A.rho = rho; A.re = re; A.accumulate = accumulate ? 1 : 0; A.finalize = finalize ? 1 : 0;
  A.outer = 1; A.inner = 1;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(shape[d] >= 1, "empty axis");
    if (d < axis) A.outer *= shape[d];
    if (d > axis) A.inner *= shape[d];
  }
  A.n = shape[axis];
  TPF_CHECK_ARG(A.n >= 3, "at least 3 nodes along the axis");
  const int64_t tot = A.outer * A.n * A.inner;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64) lowfd_kernel<double><<<blocks_for(tot), 256, 0, st>>>(A);
  else lowfd_kernel<float><<<blocks_for(tot), 256, 0, st>>>(A);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_visc_stress(int64_t n, const void* mu, const void* a, const void* b, void* out, int dtype,
                               void* stream) {
  TPF_CHECK_ARG(n >= 0 && mu && a && b && out, "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    stress_kernel<double><<<blocks_for(n), 256, 0, st>>>(n, static_cast<const double*>(mu), static_cast<const double*>(a),
                                                         static_cast<const double*>(b), static_cast<double*>(out));
  else
    stress_kernel<float><<<blocks_for(n), 256, 0, st>>>(n, static_cast<const float*>(mu), static_cast<const float*>(a),
                                                        static_cast<const float*>(b), static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_visc_accumulate(int64_t n, const void* g, int accumulate, int finalize, const void* rho, double re,
                                   void* total, int dtype, void* stream) {
  TPF_CHECK_ARG(n >= 0 && g && total && g != total, "NULL or aliased argument");
  TPF_CHECK_ARG(!finalize || (rho && re != 0.0), "finalize needs rho and a nonzero Re");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    accumulate_kernel<double><<<blocks_for(n), 256, 0, st>>>(n, static_cast<const double*>(g), accumulate, finalize,
                                                             static_cast<const double*>(rho), re,
                                                             static_cast<double*>(total));
  else
    accumulate_kernel<float><<<blocks_for(n), 256, 0, st>>>(n, static_cast<const float*>(g), accumulate, finalize,
                                                            static_cast<const float*>(rho), re,
                                                            static_cast<float*>(total));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// ---------------------------------------------------------------------------
// Interface-band form of the ccd_bulk scheme, used when psi is given
// (ViscousSpatialEvaluator.evaluate, viscous_spatial.py:50-64,158-221): inside
// the band around the interface the stress divergence with, per axis, the
// low-order derivative where that axis is the normal axis and the CCD
// derivative elsewhere; outside it mu times the CCD Laplacian; both / (Re rho).
// ---------------------------------------------------------------------------
namespace {

// NumPy's maximum: NaN if either is NaN, else the larger
__device__ __forceinline__ double np_maximum(double a, double b) {
  if (a != a || b != b) return a + b;
  return a > b ? a : b;
}

// band = core dilated by one node along every axis in turn (= the 3^ndim box
// around each node, inside the domain), core = 1e-6 < psi < 1 - 1e-6
// (_interface_band_mask, :175-187); normal[a] = (|g_a| >= max_b |g_b| and
// max > 1e-14) or max <= 1e-14, g = the low-order derivatives of psi
// (_normal_axis_masks, :189-200)
template <typename T>
__global__ void band_masks_kernel(int nd, int64_t n0, int64_t n1, int64_t n2, const T* psi, const T* g0, const T* g1,
                                  const T* g2, unsigned char* band, unsigned char* m0, unsigned char* m1,
                                  unsigned char* m2) {
  const int64_t tot = n0 * n1 * n2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k2 = i % n2, k1 = (i / n2) % n1, k0 = i / (n1 * n2);
    bool b = false;
    for (int d0 = -1; d0 <= 1 && !b; ++d0) {
      const int64_t j0 = k0 + d0;
      if (j0 < 0 || j0 >= n0) continue;
      for (int d1 = -1; d1 <= 1 && !b; ++d1) {
        const int64_t j1 = k1 + d1;
        if (j1 < 0 || j1 >= n1 || (nd < 2 && d1 != 0)) continue;
        for (int d2 = -1; d2 <= 1 && !b; ++d2) {
          const int64_t j2 = k2 + d2;
          if (j2 < 0 || j2 >= n2 || (nd < 3 && d2 != 0)) continue;
          const double p = (double)psi[(j0 * n1 + j1) * n2 + j2];
          b = (p > 1.0e-6) && (p < 1.0 - 1.0e-6);
        }
      }
    }
    band[i] = b ? 1 : 0;
    const double a0 = fabs((double)g0[i]);
    const double a1 = nd > 1 ? fabs((double)g1[i]) : 0.0;
    const double a2 = nd > 2 ? fabs((double)g2[i]) : 0.0;
    double mx = a0;
    if (nd > 1) mx = np_maximum(mx, a1);
    if (nd > 2) mx = np_maximum(mx, a2);
    const bool flat = mx <= 1.0e-14, big = mx > 1.0e-14;
    m0[i] = ((a0 >= mx && big) || flat) ? 1 : 0;
    if (nd > 1) m1[i] = ((a1 >= mx && big) || flat) ? 1 : 0;
    if (nd > 2) m2[i] = ((a2 >= mx && big) || flat) ? 1 : 0;
  }
}

// s = mask ? lo : hi (lo when mask is NULL); mode 0: out = s, 1: out += s,
// 2: out = 0 + s (the first term of a sum started from zeros)
template <typename T>
__global__ void select_kernel(int64_t n, const unsigned char* mask, const T* lo, const T* hi, int mode, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double s = (!mask || mask[i]) ? (double)lo[i] : (double)hi[i];
    if (mode == 0) out[i] = (T)s;
    else if (mode == 1) out[i] = (T)rn_add((double)out[i], s);
    else out[i] = (T)rn_add(0.0, s);
  }
}

// out = where(band, nt, mu lap) / (Re rho)
template <typename T>
__global__ void band_finalize_kernel(int64_t n, const unsigned char* band, const T* nt, const T* lap, const T* mu,
                                     const T* rho, double re, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = band[i] ? (double)nt[i] : rn_mul((double)mu[i], (double)lap[i]);
    out[i] = (T)(v / rn_mul(re, (double)rho[i]));
  }
}

}  // namespace

extern "C" int tpf_visc_band_masks(int ndim, const int64_t* shape, const void* psi, const void* const* grads,
                                   unsigned char* band, unsigned char* const* normal, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape && psi && grads && band && normal, "NULL argument or bad ndim");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  int64_t n[3] = {1, 1, 1};
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(shape[a] >= 1 && grads[a] && normal[a], "empty axis or NULL gradient / mask");
    n[a] = shape[a];
  }
  const int64_t tot = n[0] * n[1] * n[2];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* m1 = ndim > 1 ? normal[1] : nullptr;
  unsigned char* m2 = ndim > 2 ? normal[2] : nullptr;
  if (dtype == TPF_F64)
    band_masks_kernel<double><<<blocks_for(tot), 256, 0, st>>>(
        ndim, n[0], n[1], n[2], static_cast<const double*>(psi), static_cast<const double*>(grads[0]),
        ndim > 1 ? static_cast<const double*>(grads[1]) : nullptr,
        ndim > 2 ? static_cast<const double*>(grads[2]) : nullptr, band, normal[0], m1, m2);
  else
    band_masks_kernel<float><<<blocks_for(tot), 256, 0, st>>>(
        ndim, n[0], n[1], n[2], static_cast<const float*>(psi), static_cast<const float*>(grads[0]),
        ndim > 1 ? static_cast<const float*>(grads[1]) : nullptr,
        ndim > 2 ? static_cast<const float*>(grads[2]) : nullptr, band, normal[0], m1, m2);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_visc_select(int64_t n, const unsigned char* mask, const void* lo, const void* hi, int mode,
                               void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(n >= 0 && lo && out && (!mask || hi), "NULL argument");
  TPF_CHECK_ARG(mode >= 0 && mode <= 2, "mode must be 0 (set), 1 (accumulate) or 2 (zero plus)");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    select_kernel<double><<<blocks_for(n), 256, 0, st>>>(n, mask, static_cast<const double*>(lo),
                                                         static_cast<const double*>(hi), mode, static_cast<double*>(out));
  else
    select_kernel<float><<<blocks_for(n), 256, 0, st>>>(n, mask, static_cast<const float*>(lo),
                                                        static_cast<const float*>(hi), mode, static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_visc_band_finalize(int64_t n, const unsigned char* band, const void* nt, const void* lap,
                                      const void* mu, const void* rho, double re, void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(n >= 0 && band && nt && lap && mu && rho && out && re != 0.0, "NULL argument or zero Re");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    band_finalize_kernel<double><<<blocks_for(n), 256, 0, st>>>(
        n, band, static_cast<const double*>(nt), static_cast<const double*>(lap), static_cast<const double*>(mu),
        static_cast<const double*>(rho), re, static_cast<double*>(out));
  else
    band_finalize_kernel<float><<<blocks_for(n), 256, 0, st>>>(
        n, band, static_cast<const float*>(nt), static_cast<const float*>(lap), static_cast<const float*>(mu),
        static_cast<const float*>(rho), re, static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// ---------------------------------------------------------------------------
// Predictor combinations of PicardCNAdvance.advance
// (src/twophase/time_integration/cn_advance/picard_cn.py:43-96) and of the
// explicit branch of ViscousTerm.apply_cn_predictor (ns_terms/viscous.py:161-167):
//   mode 0 (forward Euler): u + dt (e / rho + vn)
//   mode 1 (trapezoid):     u + dt ((e / rho + 0.5 vn) + 0.5 vs)
//   mode 2 (Predictor.compute, explicit viscous): u + dt (e + rho vn) / rho
// ---------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void cn_combine_kernel(int64_t n, int mode, double dt, const T* u, const T* e, const T* rho, const T* vn,
                                  const T* vs, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (mode == 2) {   // explicit viscous predictor of Predictor.compute: u + dt (e + rho vn) / rho
      const double r = (double)rho[i];
      out[i] = (T)rn_add((double)u[i], rn_mul(dt, rn_add((double)e[i], rn_mul(r, (double)vn[i]))) / r);
      continue;
    }
    if (mode == 3) {   // Richardson extrapolation: (4 u_{dt/2,2} - u_dt) / 3, u = the half steps, vn = the big step
      out[i] = (T)(rn_sub(rn_mul(4.0, (double)u[i]), (double)vn[i]) / 3.0);
      continue;
    }
    const double er = (double)e[i] / (double)rho[i];
    double b;
    if (mode == 0) b = rn_add(er, (double)vn[i]);
    else b = rn_add(rn_add(er, rn_mul(0.5, (double)vn[i])), rn_mul(0.5, (double)vs[i]));
    out[i] = (T)rn_add((double)u[i], rn_mul(dt, b));
  }
}

}  // namespace

extern "C" int tpf_cn_predictor_combine(int64_t n, int mode, double dt, const void* u, const void* e, const void* rho,
                                        const void* vn, const void* vs, void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(mode >= 0 && mode <= 3,
                "mode must be 0 (forward Euler), 1 (trapezoid), 2 (explicit predictor) or 3 (Richardson)");
  TPF_CHECK_ARG(n >= 0 && u && vn && out && (mode == 3 || (e && rho)) && (mode != 1 || vs), "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    cn_combine_kernel<double><<<blocks_for(n), 256, 0, st>>>(
        n, mode, dt, static_cast<const double*>(u), static_cast<const double*>(e), static_cast<const double*>(rho),
        static_cast<const double*>(vn), static_cast<const double*>(vs), static_cast<double*>(out));
  else
    cn_combine_kernel<float><<<blocks_for(n), 256, 0, st>>>(
        n, mode, dt, static_cast<const float*>(u), static_cast<const float*>(e), static_cast<const float*>(rho),
        static_cast<const float*>(vn), static_cast<const float*>(vs), static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// ---------------------------------------------------------------------------
// Momentum predictor terms (src/twophase/time_integration/ab2_predictor.py:110-209;
// ns_terms/convection.py:43-82, gravity.py:53-86, surface_tension.py:48-96)
// ---------------------------------------------------------------------------
namespace {

// acc = (first ? 0 : acc) - u du   (ConvectionTerm: acc -= u_ax * du/dx_ax)
template <typename T>
__global__ void conv_acc_kernel(int64_t n, int first, const T* u, const T* du, T* acc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a0 = first ? 0.0 : (double)acc[i];
    acc[i] = (T)rn_sub(a0, rn_mul((double)u[i], (double)du[i]));
  }
}

// mode 0: out = -a / s (gravity, s = Fr^2); mode 1: out = (a b) / s (CSF, s = We);
// mode 2: out = a / s (the projection right-hand side div u* / dt)
template <typename T>
__global__ void scaled_kernel(int64_t n, int mode, const T* a, const T* b, double s, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (T)((mode == 0 ? -(double)a[i] : (mode == 1 ? rn_mul((double)a[i], (double)b[i]) : (double)a[i])) / s);
}

// explicit_rhs = ((rho ab2 + grav) + st) + (-gradp), ab2 = 1.5 cn - 0.5 cp (AB2)
// or cn (first step); a NULL grav / st adds +0 as the reference's zero arrays do
template <typename T>
__global__ void explicit_rhs_kernel(int64_t n, int ab2, const T* cn, const T* cp, const T* rho, const T* grav,
                                    const T* st, const T* gradp, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double c = (double)cn[i];
    if (ab2) c = (double)(T)rn_sub(rn_mul(1.5, c), rn_mul(0.5, (double)cp[i]));
    double e = rn_mul((double)rho[i], c);
    e = rn_add(e, grav ? (double)grav[i] : 0.0);
    e = rn_add(e, st ? (double)st[i] : 0.0);
    e = rn_add(e, -(double)gradp[i]);
    out[i] = (T)e;
  }
}

}  // namespace

extern "C" int tpf_ns_conv_accumulate(int64_t n, int first, const void* u, const void* du, void* acc, int dtype,
                                      void* stream) {
  TPF_CHECK_ARG(n >= 0 && u && du && acc, "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    conv_acc_kernel<double><<<blocks_for(n), 256, 0, st>>>(n, first, static_cast<const double*>(u),
                                                           static_cast<const double*>(du), static_cast<double*>(acc));
  else
    conv_acc_kernel<float><<<blocks_for(n), 256, 0, st>>>(n, first, static_cast<const float*>(u),
                                                          static_cast<const float*>(du), static_cast<float*>(acc));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_ns_scaled(int64_t n, int mode, const void* a, const void* b, double s, void* out, int dtype,
                             void* stream) {
  TPF_CHECK_ARG(mode >= 0 && mode <= 2, "mode must be 0 (gravity), 1 (CSF) or 2 (quotient)");
  TPF_CHECK_ARG(n >= 0 && a && out && (mode != 1 || b) && s != 0.0, "invalid arguments");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    scaled_kernel<double><<<blocks_for(n), 256, 0, st>>>(n, mode, static_cast<const double*>(a),
                                                         static_cast<const double*>(b), s, static_cast<double*>(out));
  else
    scaled_kernel<float><<<blocks_for(n), 256, 0, st>>>(n, mode, static_cast<const float*>(a),
                                                        static_cast<const float*>(b), s, static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_ns_explicit_rhs(int64_t n, int ab2, const void* conv_n, const void* conv_prev, const void* rho,
                                   const void* grav, const void* st_force, const void* gradp, void* out, int dtype,
                                   void* stream) {
  TPF_CHECK_ARG(n >= 0 && conv_n && rho && gradp && out && (!ab2 || conv_prev), "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    explicit_rhs_kernel<double><<<blocks_for(n), 256, 0, st>>>(
        n, ab2, static_cast<const double*>(conv_n), static_cast<const double*>(conv_prev),
        static_cast<const double*>(rho), static_cast<const double*>(grav), static_cast<const double*>(st_force),
        static_cast<const double*>(gradp), static_cast<double*>(out));
  else
    explicit_rhs_kernel<float><<<blocks_for(n), 256, 0, st>>>(
        n, ab2, static_cast<const float*>(conv_n), static_cast<const float*>(conv_prev),
        static_cast<const float*>(rho), static_cast<const float*>(grav), static_cast<const float*>(st_force),
        static_cast<const float*>(gradp), static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// Steps beside the PPE: the CFL time-step maxima (reference
// src/twophase/time_integration/cfl.py:85-137).  The velocity corrector is an
// epilogue of the CCD line kernels (tpf_ccd_apply_corrector in ccd.cu).
#include "tpf_common.cuh"

namespace {

struct CflPtrs {
  const void* comp[3];
  const void* mu;
  const void* rho;
};

// running maximum that keeps a NaN once seen (as the reference's xp.max does)
__device__ __forceinline__ void keep_max(double& m, double v) {
  if (v != v || v > m) m = v;
}

// out[c] = max_i |comp_c[i]| (c < ncomp), out[3] = max_i mu[i] / rho[i] (if mu).
// All values are >= 0 (or NaN), so the bit patterns order like the values and
// one 64-bit atomicMax per warp combines them (order-independent: exact).
template <typename T>
__global__ void cfl_maxima_kernel(int64_t n, int ncomp, CflPtrs p, unsigned long long* out) {
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (c < ncomp) keep_max(m[c], fabs((double)static_cast<const T*>(p.comp[c])[i]));
    if (p.mu)
      keep_max(m[3], (double)static_cast<const T*>(p.mu)[i] / (double)static_cast<const T*>(p.rho)[i]);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
    for (int off = 16; off > 0; off >>= 1) keep_max(m[c], __shfl_xor_sync(0xffffffffu, m[c], off));
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c < ncomp || (c == 3 && p.mu)) atomicMax(out + c, (unsigned long long)__double_as_longlong(m[c]));
  }
}

}  // namespace

extern "C" int tpf_cfl_maxima(int64_t n, int ncomp, const void* const* comps, const void* mu, const void* rho,
                              int dtype, double* out, void* stream) {
  TPF_CHECK_ARG(n >= 0, "negative size");
  TPF_CHECK_ARG(ncomp >= 1 && ncomp <= 3, "1..3 velocity components (got %d)", ncomp);
  TPF_CHECK_ARG(comps != nullptr && out != nullptr, "NULL argument");
  for (int c = 0; c < ncomp; ++c) TPF_CHECK_ARG(comps[c] != nullptr, "velocity component %d is NULL", c);
  TPF_CHECK_ARG((mu == nullptr) == (rho == nullptr), "mu and rho are given together");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TPF_CUDA_TRY(cudaMemsetAsync(out, 0, 4 * sizeof(double), s));
  if (n == 0) return TPF_OK;
  CflPtrs p{};
  for (int c = 0; c < ncomp; ++c) p.comp[c] = comps[c];
  p.mu = mu;
  p.rho = rho;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)tpf::sm_count() * 8);
  unsigned long long* o = reinterpret_cast<unsigned long long*>(out);
  if (dtype == TPF_F64) cfl_maxima_kernel<double><<<blocks, 256, 0, s>>>(n, ncomp, p, o);
  else cfl_maxima_kernel<float><<<blocks, 256, 0, s>>>(n, ncomp, p, o);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// ---- interface geometry and properties from the CLS field psi --------------------
// Reference: src/twophase/levelset/curvature.py:60-127 (DCCD filter),
// curvature_psi.py:72-173 (curvature from psi), heaviside.py:167-187
// (properties).  Products and sums use explicit round-to-nearest operations in
// the order NumPy evaluates the reference's expressions (no fused multiply-add).

namespace {

struct Shape3 {
  int64_t n[3];   // nodes per axis (n[2] = 1 in 2-D)
  int ndim;
};

__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }

// one axis of the DCCD filter (curvature.py:60-102): out = f + c (f[+1] - 2 f + f[-1])
// on nodes 1..N-1 (wall) or 0..N-1 with wrap-around and image node N <- node 0
// (periodic); every other node is copied.  c = eps, or eps * sw[node].
template <typename T>
__global__ void dccd_axis_kernel(Shape3 s, int axis, int periodic, double eps, const T* sw, const T* f, T* out) {
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  const int64_t na = s.n[axis];
  int64_t stride = 1;
  for (int a = axis + 1; a < 3; ++a) stride *= s.n[a];
  const int64_t N = na - 1;   // cells along the axis
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = (i / stride) % na;
    const double fc = (double)f[i];
    double v = fc;
    if (periodic) {
      const int64_t kk = (k == N) ? 0 : k;             // the image node takes node 0's result
      const int64_t ic = i + (kk - k) * stride;
      const double c0 = (double)f[ic];
      const double fm = (double)f[ic + (((kk == 0) ? N - 1 : kk - 1) - kk) * stride];
      const double fp = (double)f[ic + (((kk == N - 1) ? 0 : kk + 1) - kk) * stride];
      const double c = sw ? rn_mul(eps, (double)sw[ic]) : eps;
      v = rn_add(c0, rn_mul(c, rn_add(rn_sub(fp, rn_mul(2.0, c0)), fm)));
    } else if (k >= 1 && k <= N - 1) {
      const double fm = (double)f[i - stride], fp = (double)f[i + stride];
      const double c = sw ? rn_mul(eps, (double)sw[i]) : eps;
      v = rn_add(fc, rn_mul(c, rn_add(rn_sub(fp, rn_mul(2.0, fc)), fm)));
    }
    out[i] = (T)v;
  }
}

// wall axes: both boundary planes take the unfiltered input (curvature.py:118-126)
template <typename T>
__global__ void dccd_restore_kernel(Shape3 s, int axis, const T* f0, T* out) {
  const int64_t na = s.n[axis];
  int64_t stride = 1;
  for (int a = axis + 1; a < 3; ++a) stride *= s.n[a];
  const int64_t outer = (s.n[0] * s.n[1] * s.n[2]) / (na * stride);
  const int64_t tot = outer * stride * 2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t side = e / (outer * stride), r = e - side * outer * stride;
    const int64_t o = r / stride, in = r - o * stride;
    const int64_t idx = (o * na + (side ? na - 1 : 0)) * stride + in;
    out[idx] = f0[idx];
  }
}

struct CurvPtrs {
  const void* d1[3];
  const void* d2[3];
  const void* mixed[3];   // 2-D: [0] = psi_xy; 3-D: xy, xz, yz
};

// kappa from the (filtered) CCD derivatives (curvature_psi.py:72-173), zero
// where psi <= psi_min or psi >= 1 - psi_min
template <typename T>
__global__ void curvature_kernel(int ndim, int64_t n, const T* psi, CurvPtrs p, double psi_min, T* kappa) {
  const double EPS_GRAD = 1e-30;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    auto D1 = [&](int a) { return (double)static_cast<const T*>(p.d1[a])[i]; };
    auto D2 = [&](int a) { return (double)static_cast<const T*>(p.d2[a])[i]; };
    auto MX = [&](int a) { return (double)static_cast<const T*>(p.mixed[a])[i]; };
    double grad_sq = rn_mul(D1(0), D1(0));
    for (int a = 1; a < ndim; ++a) grad_sq = rn_add(grad_sq, rn_mul(D1(a), D1(a)));
    double k;
    if (ndim == 2) {
      const double px = D1(0), py = D1(1), pxx = D2(0), pyy = D2(1), pxy = MX(0);
      const double num = rn_add(rn_sub(rn_mul(rn_mul(py, py), pxx), rn_mul(rn_mul(rn_mul(2.0, px), py), pxy)),
                                rn_mul(rn_mul(px, px), pyy));
      const double cube = pow(rn_add(grad_sq, EPS_GRAD), 1.5);
      k = -num / cube;
    } else {
      const double lap = rn_add(rn_add(D2(0), D2(1)), D2(2));
      double con = rn_mul(rn_mul(D1(0), D1(0)), D2(0));
      con = rn_add(con, rn_mul(rn_mul(D1(1), D1(1)), D2(1)));
      con = rn_add(con, rn_mul(rn_mul(D1(2), D1(2)), D2(2)));
      con = rn_add(con, rn_mul(rn_mul(rn_mul(2.0, D1(0)), D1(1)), MX(0)));
      con = rn_add(con, rn_mul(rn_mul(rn_mul(2.0, D1(0)), D1(2)), MX(1)));
      con = rn_add(con, rn_mul(rn_mul(rn_mul(2.0, D1(1)), D1(2)), MX(2)));
      const double gs = rn_add(grad_sq, EPS_GRAD);
      k = -rn_sub(lap, con / gs) / sqrt(gs);
    }
    const double ps = (double)psi[i];
    if (ps <= psi_min || ps >= 1.0 - psi_min) k = 0.0;
    kappa[i] = (T)k;
  }
}

// 3x3 Gaussian [1 2 1; 2 4 2; 1 2 1] / 16 with edge replication
// (curvature_psi.py:176-197), 2-D
template <typename T>
__global__ void gaussian3x3_kernel(int64_t n0, int64_t n1, const T* in, T* out) {
  const int64_t tot = n0 * n1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t y = i / n1, x = i - y * n1;
    auto at = [&](int64_t yy, int64_t xx) {
      yy = yy < 0 ? 0 : (yy >= n0 ? n0 - 1 : yy);
      xx = xx < 0 ? 0 : (xx >= n1 ? n1 - 1 : xx);
      return (double)in[yy * n1 + xx];
    };
    double r = rn_mul(1.0, at(y - 1, x - 1));
    r = rn_add(r, rn_mul(2.0, at(y - 1, x)));
    r = rn_add(r, rn_mul(1.0, at(y - 1, x + 1)));
    r = rn_add(r, rn_mul(2.0, at(y, x - 1)));
    r = rn_add(r, rn_mul(4.0, at(y, x)));
    r = rn_add(r, rn_mul(2.0, at(y, x + 1)));
    r = rn_add(r, rn_mul(1.0, at(y + 1, x - 1)));
    r = rn_add(r, rn_mul(2.0, at(y + 1, x)));
    r = rn_add(r, rn_mul(1.0, at(y + 1, x + 1)));
    out[i] = (T)(r / 16.0);
  }
}

// rho = rho_g + (rho_l - rho_g) psi, mu = mu_g + (mu_l - mu_g) psi (heaviside.py:167-187)
template <typename T>
__global__ void properties_kernel(int64_t n, const T* psi, double rl, double rg, double ml, double mg, T* rho, T* mu) {
  const double dr = rl - rg, dm = ml - mg;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ps = (double)psi[i];
    if (rho) rho[i] = (T)rn_add(rg, rn_mul(dr, ps));
    if (mu) mu[i] = (T)rn_add(mg, rn_mul(dm, ps));
  }
}

inline int ew_blocks64(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)tpf::sm_count() * 16)); }

template <typename T>
int dccd_filter_t(const Shape3& s, const int* periodic, double eps, const void* sw, const void* f, void* out, void* tmp,
                  cudaStream_t st) {
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  const T* src = static_cast<const T*>(f);
  // ping-pong so that the last pass lands in out
  T* bufs[2] = {static_cast<T*>(s.ndim % 2 == 1 ? out : tmp), static_cast<T*>(s.ndim % 2 == 1 ? tmp : out)};
  for (int ax = 0; ax < s.ndim; ++ax) {
    T* dst = bufs[ax & 1];
    dccd_axis_kernel<T><<<ew_blocks64(tot), 256, 0, st>>>(s, ax, periodic[ax], eps, static_cast<const T*>(sw), src, dst);
    src = dst;
  }
  for (int ax = 0; ax < s.ndim; ++ax)
    if (!periodic[ax]) dccd_restore_kernel<T><<<ew_blocks64(tot), 256, 0, st>>>(s, ax, static_cast<const T*>(f), static_cast<T*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

}  // namespace

extern "C" int tpf_dccd_filter(int ndim, const int64_t* shape, const int* periodic, double eps, const void* sw,
                               const void* f, void* out, void* tmp, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim == 2 || ndim == 3, "ndim must be 2 or 3");
  TPF_CHECK_ARG(shape && periodic && f && out && tmp, "NULL argument");
  TPF_CHECK_ARG(f != out && f != tmp && out != tmp && (!sw || (sw != out && sw != tmp)),
                "the filter's input, output and workspace must be distinct");
  Shape3 s{{1, 1, 1}, ndim};
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(shape[a] >= 3, "at least 3 nodes per axis (got %lld)", (long long)shape[a]);
    s.n[a] = shape[a];
  }
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return dtype == TPF_F64 ? dccd_filter_t<double>(s, periodic, eps, sw, f, out, tmp, st)
                          : dccd_filter_t<float>(s, periodic, eps, sw, f, out, tmp, st);
}

extern "C" int tpf_curvature_psi(int ndim, int64_t n, const void* psi, const void* const* d1, const void* const* d2,
                                 const void* const* mixed, double psi_min, void* kappa, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim == 2 || ndim == 3, "ndim must be 2 or 3");
  TPF_CHECK_ARG(n >= 0 && psi && d1 && d2 && mixed && kappa, "NULL argument");
  CurvPtrs p{};
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(d1[a] && d2[a], "derivative %d is NULL", a);
    p.d1[a] = d1[a];
    p.d2[a] = d2[a];
  }
  const int nm = ndim == 2 ? 1 : 3;
  for (int a = 0; a < nm; ++a) {
    TPF_CHECK_ARG(mixed[a], "mixed derivative %d is NULL", a);
    p.mixed[a] = mixed[a];
  }
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) return TPF_OK;
  if (dtype == TPF_F64)
    curvature_kernel<double><<<ew_blocks64(n), 256, 0, st>>>(ndim, n, static_cast<const double*>(psi), p, psi_min,
                                                             static_cast<double*>(kappa));
  else
    curvature_kernel<float><<<ew_blocks64(n), 256, 0, st>>>(ndim, n, static_cast<const float*>(psi), p, psi_min,
                                                            static_cast<float*>(kappa));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_gaussian3x3(int64_t n0, int64_t n1, const void* in, void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(n0 >= 1 && n1 >= 1 && in && out && in != out, "invalid arguments");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    gaussian3x3_kernel<double><<<ew_blocks64(n0 * n1), 256, 0, st>>>(n0, n1, static_cast<const double*>(in),
                                                                     static_cast<double*>(out));
  else
    gaussian3x3_kernel<float><<<ew_blocks64(n0 * n1), 256, 0, st>>>(n0, n1, static_cast<const float*>(in),
                                                                    static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_update_properties(int64_t n, const void* psi, double rho_l, double rho_g, double mu_l, double mu_g,
                                     void* rho, void* mu, int dtype, void* stream) {
  TPF_CHECK_ARG(n >= 0 && psi && (rho || mu), "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) return TPF_OK;
  if (dtype == TPF_F64)
    properties_kernel<double><<<ew_blocks64(n), 256, 0, st>>>(n, static_cast<const double*>(psi), rho_l, rho_g, mu_l,
                                                              mu_g, static_cast<double*>(rho), static_cast<double*>(mu));
  else
    properties_kernel<float><<<ew_blocks64(n), 256, 0, st>>>(n, static_cast<const float*>(psi), rho_l, rho_g, mu_l,
                                                             mu_g, static_cast<float*>(rho), static_cast<float*>(mu));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

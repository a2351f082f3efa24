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
template <typename T, int ND>
__global__ void curvature_kernel(int64_t n, const T* psi, CurvPtrs p, double psi_min, T* kappa) {
  const double EPS_GRAD = 1e-30;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    auto D1 = [&](int a) { return (double)static_cast<const T*>(p.d1[a])[i]; };
    auto D2 = [&](int a) { return (double)static_cast<const T*>(p.d2[a])[i]; };
    auto MX = [&](int a) { return (double)static_cast<const T*>(p.mixed[a])[i]; };
    double grad_sq = rn_mul(D1(0), D1(0));
#pragma unroll
    for (int a = 1; a < ND; ++a) grad_sq = rn_add(grad_sq, rn_mul(D1(a), D1(a)));
    double k;
    if (ND == 2) {
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

// The DCCD filter (curvature.py:60-127): per axis in turn
// out = f + c (f[+1] - 2 f + f[-1]) on nodes 1..N-1 (wall) or 0..N-1 with
// wrap-around and image node N <- node 0 (periodic), c = eps or eps * sw[node];
// every other node is copied.  2-D: both axis passes in one kernel.  A block owns a TI x TJ x TK
// tile of outputs; it stages f on the tile plus one node on each side (the
// coordinates of a periodic axis taken modulo N, so node N reads node 0 and
// the halo wraps), forms the axis-0 pass on TI x (TJ+2) x (TK+2) nodes, the
// axis-1 pass on TI x TJ x (TK+2), the axis-2 pass on the tile, all in shared
// memory, then restores the wall planes from f.  Each pass rounds to T like
// the reference's array passes; coefficients are read at the coordinates the
// reference uses (a periodic image plane of an earlier axis keeps its own
// coefficient).  Used for 2-D (K3 = false: TK = 1, no axis-2 pass).
template <typename T, int TI, int TJ, int TK, bool K3>
__global__ void __launch_bounds__(256) dccd_fused_kernel(Shape3 s, int p0, int p1, int p2, double eps, const T* sw,
                                                         const T* f, T* out) {
  constexpr int HK = K3 ? 1 : 0;
  constexpr int EI = TI + 2, EJ = TJ + 2, EK = TK + 2 * HK;
  __shared__ double F[EI][EJ][EK];
  __shared__ double X[TI][EJ][EK];
  __shared__ double Y[TI][TJ][EK];
  const int64_t n0 = s.n[0], n1 = s.n[1], n2 = s.n[2];
  const int64_t N0 = n0 - 1, N1 = n1 - 1, N2 = n2 - 1;
  const int64_t c0 = (n0 + TI - 1) / TI, c1 = (n1 + TJ - 1) / TJ, c2 = K3 ? (n2 + TK - 1) / TK : 1;
  auto W = [](int64_t x, int64_t N, int per) -> int64_t {
    return per ? ((x % N) + N) % N : (x < 0 ? 0 : (x > N ? N : x));
  };
  auto coef = [&](int64_t i, int64_t j, int64_t k) -> double {
    return sw ? rn_mul(eps, (double)sw[(i * n1 + j) * n2 + k]) : eps;
  };
  const int64_t tiles = c0 * c1 * c2;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t tk = tile % c2, tj = (tile / c2) % c1, ti = tile / (c1 * c2);
    const int64_t i0 = ti * TI, j0 = tj * TJ, k0 = tk * TK;
    for (int e = threadIdx.x; e < EI * EJ * EK; e += blockDim.x) {
      const int a = e / (EJ * EK), b = (e / EK) % EJ, c = e % EK;
      const int64_t gi = W(i0 - 1 + a, N0, p0), gj = W(j0 - 1 + b, N1, p1);
      const int64_t gk = K3 ? W(k0 - 1 + c, N2, p2) : 0;
      F[a][b][c] = (double)f[(gi * n1 + gj) * n2 + gk];
    }
    __syncthreads();
    // axis 0 at (raw i, node W(j), node W(k))
    for (int e = threadIdx.x; e < TI * EJ * EK; e += blockDim.x) {
      const int a = e / (EJ * EK), b = (e / EK) % EJ, c = e % EK;
      const int64_t i = i0 + a;
      if (i > N0) continue;
      double v = F[a + 1][b][c];
      if (p0 || (i >= 1 && i <= N0 - 1)) {
        const int64_t ci = (p0 && i == N0) ? 0 : i;
        const int64_t gj = W(j0 - 1 + b, N1, p1), gk = K3 ? W(k0 - 1 + c, N2, p2) : 0;
        v = rn_add(v, rn_mul(coef(ci, gj, gk), rn_add(rn_sub(F[a + 2][b][c], rn_mul(2.0, v)), F[a][b][c])));
      }
      X[a][b][c] = (double)(T)v;
    }
    __syncthreads();
    // axis 1 at (raw i, raw j, node W(k))
    for (int e = threadIdx.x; e < TI * TJ * EK; e += blockDim.x) {
      const int a = e / (TJ * EK), b = (e / EK) % TJ, c = e % EK;
      const int64_t i = i0 + a, j = j0 + b;
      if (i > N0 || j > N1) continue;
      double v = X[a][b + 1][c];
      if (p1 || (j >= 1 && j <= N1 - 1)) {
        const int64_t cj = (p1 && j == N1) ? 0 : j;
        const int64_t gk = K3 ? W(k0 - 1 + c, N2, p2) : 0;
        v = rn_add(v, rn_mul(coef(i, cj, gk), rn_add(rn_sub(X[a][b + 2][c], rn_mul(2.0, v)), X[a][b][c])));
      }
      Y[a][b][c] = (double)(T)v;
    }
    __syncthreads();
    // axis 2 at (raw i, raw j, raw k), then the wall planes take f
    for (int e = threadIdx.x; e < TI * TJ * TK; e += blockDim.x) {
      const int a = e / (TJ * TK), b = (e / TK) % TJ, c = e % TK;
      const int64_t i = i0 + a, j = j0 + b, k = k0 + c;
      if (i > N0 || j > N1 || (K3 && k > N2)) continue;
      double v = Y[a][b][c + HK];
      if (K3 && (p2 || (k >= 1 && k <= N2 - 1))) {
        const int64_t ck = (p2 && k == N2) ? 0 : k;
        v = rn_add(v, rn_mul(coef(i, j, ck), rn_add(rn_sub(Y[a][b][c + 2], rn_mul(2.0, v)), Y[a][b][c])));
      }
      const int64_t idx = (i * n1 + j) * n2 + k;
      const bool wall_plane = (!p0 && (i == 0 || i == N0)) || (!p1 && (j == 0 || j == N1)) ||
                              (K3 && !p2 && (k == 0 || k == N2));
      out[idx] = wall_plane ? f[idx] : (T)v;
    }
    __syncthreads();
  }
}

template <typename T>
int dccd_filter_t(const Shape3& s, const int* periodic, double eps, const void* sw, const void* f, void* out, void* tmp,
                  cudaStream_t st) {
  const int64_t sms = tpf::sm_count();
  const T* swp = static_cast<const T*>(sw);
  const T* fp = static_cast<const T*>(f);
  if (s.ndim == 2) {   // both passes in one tiled kernel
    constexpr int TI = 8, TJ = 64;
    const int64_t tiles = ((s.n[0] + TI - 1) / TI) * ((s.n[1] + TJ - 1) / TJ);
    dccd_fused_kernel<T, TI, TJ, 1, false><<<(int)std::min<int64_t>(tiles, sms * 8), 256, 0, st>>>(
        s, periodic[0], periodic[1], 0, eps, swp, fp, static_cast<T*>(out));
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  }
  // 3-D: one streaming kernel per axis (ping-pong so that the last pass lands
  // in out), then the wall planes.  A tiled all-axes kernel was slower here:
  // per-tile barriers and halo staging left it latency-bound.
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  const T* src = fp;
  T* bufs[2] = {static_cast<T*>(out), static_cast<T*>(tmp)};
  for (int ax = 0; ax < 3; ++ax) {
    T* dst = bufs[ax & 1];
    dccd_axis_kernel<T><<<ew_blocks64(tot), 256, 0, st>>>(s, ax, periodic[ax], eps, swp, src, dst);
    src = dst;
  }
  for (int ax = 0; ax < 3; ++ax)
    if (!periodic[ax]) dccd_restore_kernel<T><<<ew_blocks64(tot), 256, 0, st>>>(s, ax, fp, static_cast<T*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

}  // namespace

extern "C" int tpf_dccd_filter(int ndim, const int64_t* shape, const int* periodic, double eps, const void* sw,
                               const void* f, void* out, void* tmp, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim == 2 || ndim == 3, "ndim must be 2 or 3");
  TPF_CHECK_ARG(shape && periodic && f && out, "NULL argument");
  TPF_CHECK_ARG(ndim == 2 || tmp, "a 3-D filter needs the workspace tmp");
  TPF_CHECK_ARG(f != out && (!sw || sw != out) && (ndim == 2 || (tmp != f && tmp != out && tmp != sw)),
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
  const int nb = ew_blocks64(n);
  if (dtype == TPF_F64) {
    const double* ps = static_cast<const double*>(psi);
    double* kp = static_cast<double*>(kappa);
    if (ndim == 2) curvature_kernel<double, 2><<<nb, 256, 0, st>>>(n, ps, p, psi_min, kp);
    else curvature_kernel<double, 3><<<nb, 256, 0, st>>>(n, ps, p, psi_min, kp);
  } else {
    const float* ps = static_cast<const float*>(psi);
    float* kp = static_cast<float*>(kappa);
    if (ndim == 2) curvature_kernel<float, 2><<<nb, 256, 0, st>>>(n, ps, p, psi_min, kp);
    else curvature_kernel<float, 3><<<nb, 256, 0, st>>>(n, ps, p, psi_min, kp);
  }
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

// ---------------------------------------------------------------------------
// Rhie-Chow face-velocity divergence along one axis
// (RhieChowInterpolator.face_velocity_divergence, src/twophase/spatial/rhie_chow.py:55-284)
//
// face j (between nodes j-1 and j), j = 1..N:
//   u_f = 0.5 (u_{j-1} + u_j) - (dt * 2 / (rho_{j-1} + rho_j)) * bracket,
//   bracket = (p_j - p_{j-1}) / h - 0.5 (dp_{j-1} + dp_j)
//             [ - (0.5 (kappa_{j-1} + kappa_j) (psi_j - psi_{j-1}) / (h We) - 0.5 (fs_{j-1} + fs_j)) ]
// face 0: 0 on a wall axis; nodes (N, 0) on a periodic axis.  On a wall axis
// the boundary nodes' dp (and fs) are one-sided differences.
// div_k = (u_f[k+1] - u_f[k]) / h, k < N; node N: -u_f[N] / h (wall) or
// (u_f[0] - u_f[N]) / h (periodic).  Each thread recomputes its node's two
// faces from the neighbours (L1/L2 hits) in the reference's operation order
// on a contiguous axis; on a strided axis one thread marches along each line.
// ---------------------------------------------------------------------------
namespace {

struct RcArgs {
  const void *u, *p, *rho, *dp, *kappa, *psi, *dpsi;
  void* out;
  int64_t outer, n, inner;
  double h, dt, we;
  int periodic, bf, accumulate;
};

template <typename T>
__device__ __forceinline__ double ld(const void* a, int64_t i) { return (double)static_cast<const T*>(a)[i]; }

template <typename T>
__device__ __forceinline__ double rc_dp(const RcArgs& a, int64_t base, int64_t m) {
  const int64_t N = a.n - 1, s = a.inner;
  if (!a.periodic && m == 0) return rn_sub(ld<T>(a.p, base + s), ld<T>(a.p, base)) / a.h;
  if (!a.periodic && m == N) return rn_sub(ld<T>(a.p, base + N * s), ld<T>(a.p, base + (N - 1) * s)) / a.h;
  return ld<T>(a.dp, base + m * s);
}

template <typename T>
__device__ __forceinline__ double rc_fs(const RcArgs& a, int64_t base, int64_t m) {
  const int64_t N = a.n - 1, s = a.inner;
  const double hw = rn_mul(a.h, a.we);
  if (!a.periodic && m == 0)
    return rn_mul(ld<T>(a.kappa, base), rn_sub(ld<T>(a.psi, base + s), ld<T>(a.psi, base))) / hw;
  if (!a.periodic && m == N)
    return rn_mul(ld<T>(a.kappa, base + N * s), rn_sub(ld<T>(a.psi, base + N * s), ld<T>(a.psi, base + (N - 1) * s))) / hw;
  return rn_mul(ld<T>(a.kappa, base + m * s), ld<T>(a.dpsi, base + m * s)) / a.we;
}

// face velocity between nodes l and r of the line starting at base
template <typename T>
__device__ __forceinline__ double rc_face(const RcArgs& a, int64_t base, int64_t l, int64_t r) {
  const int64_t s = a.inner;
  const int64_t il = base + l * s, ir = base + r * s;
  const double ubar = rn_mul(0.5, rn_add(ld<T>(a.u, il), ld<T>(a.u, ir)));
  const double dpf = rn_sub(ld<T>(a.p, ir), ld<T>(a.p, il)) / a.h;
  const double dpb = rn_mul(0.5, rn_add(rc_dp<T>(a, base, l), rc_dp<T>(a, base, r)));
  const double inv = 2.0 / rn_add(ld<T>(a.rho, il), ld<T>(a.rho, ir));
  double br = rn_sub(dpf, dpb);
  if (a.bf) {
    const double kf = rn_mul(0.5, rn_add(ld<T>(a.kappa, il), ld<T>(a.kappa, ir)));
    const double fsf = rn_mul(kf, rn_sub(ld<T>(a.psi, ir), ld<T>(a.psi, il))) / rn_mul(a.h, a.we);
    const double fsb = rn_mul(0.5, rn_add(rc_fs<T>(a, base, l), rc_fs<T>(a, base, r)));
    br = rn_sub(br, rn_sub(fsf, fsb));
  }
  return rn_sub(ubar, rn_mul(rn_mul(a.dt, inv), br));
}

template <typename T>
__global__ void rc_divergence_kernel(RcArgs a) {
  const int64_t tot = a.outer * a.n * a.inner;
  const int64_t N = a.n - 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t in = i % a.inner;
    const int64_t k = (i / a.inner) % a.n;
    const int64_t o = i / (a.inner * a.n);
    const int64_t base = o * a.n * a.inner + in;
    // face 0: 0 on a wall axis, the wrap-around face on a periodic one
    auto face = [&](int64_t j) -> double {
      if (j == 0) return a.periodic ? rc_face<T>(a, base, N, 0) : 0.0;
      return rc_face<T>(a, base, j - 1, j);
    };
    double d;
    if (k < N)
      d = rn_sub(face(k + 1), face(k)) / a.h;
    else
      d = a.periodic ? rn_sub(face(0), face(N)) / a.h : (-face(N)) / a.h;
    T* out = static_cast<T*>(a.out);
    out[i] = (T)(a.accumulate ? rn_add((double)out[i], d) : rn_add(0.0, d));
  }
}

// one node's operands; dpe / fse are the effective cell values (one-sided on
// the wall planes)
struct RcNode {
  double u, p, rho, dp, kap, psi, dpsi, dpe, fse;
};

template <typename T, bool BF>
__device__ __forceinline__ RcNode rc_load(const RcArgs& a, int64_t idx) {
  RcNode v;
  v.u = ld<T>(a.u, idx);
  v.p = ld<T>(a.p, idx);
  v.rho = ld<T>(a.rho, idx);
  v.dp = ld<T>(a.dp, idx);
  if (BF) {
    v.kap = ld<T>(a.kappa, idx);
    v.psi = ld<T>(a.psi, idx);
    v.dpsi = ld<T>(a.dpsi, idx);
  } else {
    v.kap = v.psi = v.dpsi = 0.0;
  }
  v.dpe = v.dp;
  v.fse = 0.0;
  return v;
}

template <bool BF>
__device__ __forceinline__ double rc_face_nodes(const RcArgs& a, const RcNode& l, const RcNode& r) {
  const double ubar = rn_mul(0.5, rn_add(l.u, r.u));
  const double dpf = rn_sub(r.p, l.p) / a.h;
  const double dpb = rn_mul(0.5, rn_add(l.dpe, r.dpe));
  const double inv = 2.0 / rn_add(l.rho, r.rho);
  double br = rn_sub(dpf, dpb);
  if (BF) {
    const double kf = rn_mul(0.5, rn_add(l.kap, r.kap));
    const double fsf = rn_mul(kf, rn_sub(r.psi, l.psi)) / rn_mul(a.h, a.we);
    const double fsb = rn_mul(0.5, rn_add(l.fse, r.fse));
    br = rn_sub(br, rn_sub(fsf, fsb));
  }
  return rn_sub(ubar, rn_mul(rn_mul(a.dt, inv), br));
}

// operands of node m of the line at base with its effective cell values
// (one-sided differences on the wall planes, curvature force kappa D1psi / We)
template <typename T, bool BF>
__device__ __forceinline__ RcNode rc_load_eff(const RcArgs& a, int64_t base, int64_t m) {
  const int64_t N = a.n - 1, s = a.inner;
  RcNode v = rc_load<T, BF>(a, base + m * s);
  const bool lo = !a.periodic && m == 0, hi = !a.periodic && m == N;
  if (lo || hi) {
    const int64_t nb = base + (lo ? 1 : N - 1) * s;
    const double pn = ld<T>(a.p, nb);
    v.dpe = (lo ? rn_sub(pn, v.p) : rn_sub(v.p, pn)) / a.h;
    if (BF) {
      const double sn = ld<T>(a.psi, nb);
      v.fse = rn_mul(v.kap, lo ? rn_sub(sn, v.psi) : rn_sub(v.psi, sn)) / rn_mul(a.h, a.we);
    }
  } else if (BF) {
    v.fse = rn_mul(v.kap, v.dpsi) / a.we;
  }
  return v;
}

// face j of a line (j = 0: 0 on a wall axis, nodes (N, 0) on a periodic one)
template <typename T, bool BF>
__device__ __forceinline__ double rc_face_j(const RcArgs& a, int64_t base, int64_t j) {
  if (j == 0) {
    if (!a.periodic) return 0.0;
    return rc_face_nodes<BF>(a, rc_load_eff<T, BF>(a, base, a.n - 1), rc_load_eff<T, BF>(a, base, 0));
  }
  return rc_face_nodes<BF>(a, rc_load_eff<T, BF>(a, base, j - 1), rc_load_eff<T, BF>(a, base, j));
}

template <typename T>
__device__ __forceinline__ void rc_store(const RcArgs& a, int64_t idx, double d) {
  T* out = static_cast<T*>(a.out);
  out[idx] = (T)(a.accumulate ? rn_add((double)out[idx], d) : rn_add(0.0, d));
}

// Strided axis: thread (chunk q, line c) marches over nodes [q C, q C + C) of
// line c, each node loaded once and each face formed once, the chunk's first
// face from its left neighbour.  Consecutive threads take consecutive lines
// (consecutive inner indices), so every load of a step is coalesced.
template <typename T, bool BF>
__global__ void __launch_bounds__(256) rc_march_kernel(RcArgs a, int64_t chunk, int64_t nchunks) {
  const int64_t lines = a.outer * a.inner;
  const int64_t N = a.n - 1, s = a.inner;
  const int64_t work = lines * nchunks;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < work; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / lines, c = t - q * lines;
    const int64_t o = c / s, in = c - o * s;
    const int64_t base = o * a.n * s + in;
    const int64_t k0 = q * chunk, k1 = min(k0 + chunk, a.n);   // nodes [k0, k1)
    double fprev = rc_face_j<T, BF>(a, base, k0);
    RcNode cur = rc_load_eff<T, BF>(a, base, k0);
    RcNode nxt = rc_load_eff<T, BF>(a, base, k0 < N ? k0 + 1 : k0);
    for (int64_t k = k0; k < k1; ++k) {
      if (k < N) {
        // the node after next and this node's running sum are loaded before
        // the store: the compiler cannot prove that the output overlaps no
        // input, so a load placed after the store would wait for it
        const RcNode nn = rc_load_eff<T, BF>(a, base, k + 2 <= N ? k + 2 : N);
        const double old = a.accumulate ? (double)static_cast<const T*>(a.out)[base + k * s] : 0.0;
        const double f1 = rc_face_nodes<BF>(a, cur, nxt);
        const double d = rn_sub(f1, fprev) / a.h;
        static_cast<T*>(a.out)[base + k * s] = (T)rn_add(old, d);
        fprev = f1;
        cur = nxt;
        nxt = nn;
      } else {
        const double d = a.periodic ? rn_sub(rc_face_j<T, BF>(a, base, 0), fprev) / a.h : (-fprev) / a.h;
        rc_store<T>(a, base + k * s, d);
      }
    }
  }
}

// Contiguous axis (inner = 1): a block stages RC_TILE consecutive nodes plus
// one on each side in shared memory (coalesced), forms the face to the left
// of every staged node once, then the divergence of each node from two faces.
// Tiles may straddle lines; a line's wrap-around face is formed from global
// memory (once per line end).
constexpr int RC_TILE = 512;

template <typename T, bool BF>
__global__ void __launch_bounds__(256) rc_tile_kernel(RcArgs a) {
  __shared__ double su[RC_TILE + 2], sp[RC_TILE + 2], srho[RC_TILE + 2], sdpe[RC_TILE + 2];
  __shared__ double skap[BF ? RC_TILE + 2 : 1], spsi[BF ? RC_TILE + 2 : 1], sfse[BF ? RC_TILE + 2 : 1];
  __shared__ double sface[RC_TILE + 1];
  __shared__ int64_t sk[RC_TILE + 2];   // node index along the line of each slot
  const int64_t tot = a.outer * a.n;
  const int64_t n = a.n, N = a.n - 1;
  const bool small = tot < (int64_t(1) << 31);
  const int64_t ntiles = (tot + RC_TILE - 1) / RC_TILE;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t e0 = tile * RC_TILE;
    // stage nodes e0-1 .. e0+RC_TILE (slot j holds node e0-1+j)
    for (int j = threadIdx.x; j < RC_TILE + 2; j += blockDim.x) {
      const int64_t e = e0 - 1 + j;
      if (e < 0 || e >= tot) continue;
      const int64_t k = small ? (int64_t)((uint32_t)e % (uint32_t)n) : e % n;
      sk[j] = k;
      const RcNode v = rc_load_eff<T, BF>(a, e - k, k);
      su[j] = v.u; sp[j] = v.p; srho[j] = v.rho; sdpe[j] = v.dpe;
      if (BF) { skap[j] = v.kap; spsi[j] = v.psi; sfse[j] = v.fse; }
    }
    __syncthreads();
    // face to the left of node e0+j (slots j, j+1), j = 0..RC_TILE
    for (int j = threadIdx.x; j <= RC_TILE; j += blockDim.x) {
      const int64_t e = e0 + j;
      if (e >= tot) continue;
      const int64_t k = sk[j + 1];
      double f;
      if (k == 0) {
        f = rc_face_j<T, BF>(a, e, 0);
      } else {
        RcNode l, r;
        l.u = su[j]; l.p = sp[j]; l.rho = srho[j]; l.dpe = sdpe[j];
        r.u = su[j + 1]; r.p = sp[j + 1]; r.rho = srho[j + 1]; r.dpe = sdpe[j + 1];
        if (BF) {
          l.kap = skap[j]; l.psi = spsi[j]; l.fse = sfse[j];
          r.kap = skap[j + 1]; r.psi = spsi[j + 1]; r.fse = sfse[j + 1];
        }
        f = rc_face_nodes<BF>(a, l, r);
      }
      sface[j] = f;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < RC_TILE; j += blockDim.x) {
      const int64_t e = e0 + j;
      if (e >= tot) continue;
      const int64_t k = sk[j + 1];
      double d;
      if (k < N)
        d = rn_sub(sface[j + 1], sface[j]) / a.h;
      else
        d = a.periodic ? rn_sub(rc_face_j<T, BF>(a, e - k, 0), sface[j]) / a.h : (-sface[j]) / a.h;
      rc_store<T>(a, e, d);
    }
    __syncthreads();
  }
}

template <typename T, bool BF>
void launch_rc_t(const RcArgs& a, cudaStream_t st) {
  const int64_t tot = a.outer * a.n * a.inner;
  const int64_t sms = tpf::sm_count();
  if (a.inner == 1) {
    const int64_t ntiles = (tot + RC_TILE - 1) / RC_TILE;
    rc_tile_kernel<T, BF><<<(int)std::max<int64_t>(1, std::min<int64_t>(ntiles, sms * 8)), 256, 0, st>>>(a);
  } else if (a.inner >= 32) {
    // chunk length: autotuned among kChunks (the march gives the same values
    // for every chunk length), else enough threads to fill the GPU (about
    // 2048 per SM), 8..64 nodes
    const int64_t lines = a.outer * a.inner;
    int64_t chunk = (lines * a.n) / (sms * 2048);
    chunk = std::max<int64_t>(8, std::min<int64_t>(64, chunk));
    static constexpr int64_t kChunks[5] = {8, 16, 32, 64, 128};
    auto launch = [&](int64_t ck, void* out, cudaStream_t s2) -> int {
      RcArgs b = a;
      b.out = out;
      const int64_t nchunks = (a.n + ck - 1) / ck;
      const int64_t work = lines * nchunks;
      const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, sms * 8));
      rc_march_kernel<T, BF><<<blocks, 256, 0, s2>>>(b, ck, nchunks);
      return cudaPeekAtLastError() == cudaSuccess ? TPF_OK : TPF_ECUDA;
    };
    auto cand = [&](int c, void* scratch, cudaStream_t s2) { return launch(kChunks[c], scratch, s2); };
    const tpf::TuneKey key{tpf::kTuneRcMarch, (int)sizeof(T) + (BF ? 16 : 0),
                           {a.outer, a.n, a.inner, 2 * a.periodic + a.accumulate}};
    const int pick = tpf::tuned_choice(key, 5, -1, (size_t)tot * sizeof(T), st, cand);
    launch(pick >= 0 ? kChunks[pick] : chunk, a.out, st);
  } else {
    rc_divergence_kernel<T><<<ew_blocks64(tot), 256, 0, st>>>(a);
  }
}

template <typename T>
void launch_rc(const RcArgs& a, cudaStream_t st) {
  if (a.bf)
    launch_rc_t<T, true>(a, st);
  else
    launch_rc_t<T, false>(a, st);
}

}  // namespace

extern "C" int tpf_rc_divergence_axis(int ndim, const int64_t* shape, int axis, int periodic, double h, double dt,
                                      const void* u_star, const void* p, const void* rho, const void* dp,
                                      const void* kappa, const void* psi, const void* dpsi, double we,
                                      int accumulate, void* div, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3, "ndim must be 1..3");
  TPF_CHECK_ARG(shape && axis >= 0 && axis < ndim, "invalid shape or axis");
  TPF_CHECK_ARG(u_star && p && rho && dp && div, "NULL argument");
  const int bf = (kappa || psi || dpsi) ? 1 : 0;
  TPF_CHECK_ARG(!bf || (kappa && psi && dpsi && we != 0.0),
                "the balanced-force terms need kappa, psi, dpsi and a nonzero We together");
  TPF_CHECK_ARG(h > 0.0, "h must be positive");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  RcArgs a{};
  a.u = u_star; a.p = p; a.rho = rho; a.dp = dp; a.kappa = kappa; a.psi = psi; a.dpsi = dpsi; a.out = div;
  a.outer = 1; a.inner = 1;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(shape[d] >= 1, "empty axis");
    if (d < axis) a.outer *= shape[d];
    if (d > axis) a.inner *= shape[d];
  }
  a.n = shape[axis];
  TPF_CHECK_ARG(a.n >= 2, "at least 2 nodes along the axis (got %lld)", (long long)a.n);
  a.h = h; a.dt = dt; a.we = we; a.periodic = periodic ? 1 : 0; a.bf = bf; a.accumulate = accumulate ? 1 : 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    launch_rc<double>(a, st);
  else
    launch_rc<float>(a, st);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

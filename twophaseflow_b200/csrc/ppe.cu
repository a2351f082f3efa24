// Variable-density FVM pressure-Poisson solve for sm_100a.
//
// Operator (reference src/twophase/ppe/fvm_matrixfree.py:281-300,
// fvm_matrixfree_helpers.py:46-73): harmonic face coefficient
// cf = 2/(rho_L + rho_R)/d_face, L p = sum_a [cf(i-e_a)(p_{i-e_a}-p_i) +
// cf(i)(p_{i+e_a}-p_i)] / dv_a, pinned row out[pin] = p[pin].
// The CG route solves the control-volume-weighted SPD system S p = -W rhs,
// S = -W L with column/row pin (fvm_matrixfree.py:167-215), whose symmetric
// face couplings s_a = cf * prod_{b != a} dv_b are stored per face.
//
// Kernels:
//  * prepare: face couplings (FP64 + FP32 copies), Jacobi diagonals, shifted
//    line-preconditioner coefficients and their Thomas factors.
//  * persistent cooperative PCG: the whole Jacobi-PCG loop of SciPy's cg
//    (restated: stop when ||r|| < tol ||b|| at the top of an iteration) runs in
//    ONE launch; two grid-wide reductions per iteration through a bounded grid
//    barrier, the p-update is fused into the stencil (neighbour p_new values
//    are recomputed from z and p_old), scalars never leave the device.
//  * mixed precision: the same loop in FP32 (dots in FP64) as the inner solve
//    of an FP64 iterative-refinement loop, also one launch.
//  * GMRES (SciPy's left-preconditioned restarted GMRES with its gh-8400
//    inner tolerance control) driven from the host with the Hessenberg /
//    Givens state on the device; classical Gram-Schmidt with
//    re-orthogonalization replaces modified Gram-Schmidt.
#include "tpf_common.cuh"
#include "ppe_view.cuh"
#include "gmres.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <memory>
#include <vector>

namespace {

constexpr int kThreads = 512;
constexpr long long kSpinLimit = 4000000;  // polls per barrier wait (~seconds)

struct Grid3 {
  int n0, n1, n2;   // nodes per axis (n2 = 1 in 2-D)
  int N0, N1, N2;   // cells per axis (N2 = 0 in 2-D)
  int st0;          // n1 * n2
  int ndof;
  int pin;
};

__device__ __forceinline__ void coords3(const Grid3& g, int idx, int& i0, int& i1, int& i2) {
  i0 = idx / g.st0;
  int r = idx - i0 * g.st0;
  i1 = r / g.n2;
  i2 = r - i1 * g.n2;
}

// Block-contiguous node ownership for the persistent kernels: block b owns
// [b*chunk, (b+1)*chunk), thread t visits start+t, start+t+blockDim, ...; the
// (i0, i1, i2) coordinates advance incrementally (no division per node).
struct NodeIter {
  int idx, end, i0, i1, i2, d0, d1, d2;
  __device__ __forceinline__ NodeIter(const Grid3& g) : NodeIter(g, blockIdx.x, gridDim.x) {}
  // vb / nvb: this block's index and the block count of its (sub-)grid
  __device__ __forceinline__ NodeIter(const Grid3& g, int vb, int nvb) {
    const int chunk = (g.ndof + nvb - 1) / nvb;
    const int start = vb * chunk;
    end = min(start + chunk, g.ndof);
    idx = start + threadIdx.x;
    coords3(g, idx, i0, i1, i2);
    const int step = blockDim.x;
    d2 = step % g.n2;
    d1 = (step / g.n2) % g.n1;
    d0 = step / g.st0;
  }
  __device__ __forceinline__ bool ok() const { return idx < end; }
  __device__ __forceinline__ void next(const Grid3& g) {
    idx += blockDim.x;
    i2 += d2;
    if (i2 >= g.n2) { i2 -= g.n2; ++i1; }
    i1 += d1;
    if (i1 >= g.n1) { i1 -= g.n1; ++i0; }
    i0 += d0;
  }
};

struct Geo {
  const double* dv[3];     // node control-volume widths
  const double* dface[3];  // face widths
};

// S p at node idx (pin column treated as zero when ZERO_PIN, pin row identity
// handled by the caller).  s[a] are the symmetric face couplings.
template <typename T, typename PF>
__device__ __forceinline__ void s_row(const Grid3& g, int idx, int i0, int i1, int i2,
                                      const T* __restrict__ s0, const T* __restrict__ s1,
                                      const T* __restrict__ s2, PF pv, T& diag, T& off) {
  // branch-free: clamp the neighbour indices, load unconditionally, mask the
  // couplings of faces that do not exist (upper faces already store 0)
  const int m0 = (i0 > 0) ? idx - g.st0 : idx, p0 = (i0 < g.N0) ? idx + g.st0 : idx;
  const int m1 = (i1 > 0) ? idx - g.n2 : idx, p1 = (i1 < g.N1) ? idx + g.n2 : idx;
  const T sm0 = (i0 > 0) ? s0[m0] : T(0), sp0 = s0[idx];
  const T sm1 = (i1 > 0) ? s1[m1] : T(0), sp1 = s1[idx];
  T d = (sm0 + sp0) + (sm1 + sp1);
  T acc = sm0 * pv(m0) + sp0 * pv(p0) + sm1 * pv(m1) + sp1 * pv(p1);
  if (g.N2 > 0) {
    const int m2 = (i2 > 0) ? idx - 1 : idx, p2 = (i2 < g.N2) ? idx + 1 : idx;
    const T sm2 = (i2 > 0) ? s2[m2] : T(0), sp2 = s2[idx];
    d += sm2 + sp2;
    acc += sm2 * pv(m2) + sp2 * pv(p2);
  }
  diag = d;
  off = acc;
}

// ---- prepare ---------------------------------------------------------------

struct PrepArgs {
  Grid3 g;
  Geo geo;
  const double* rho;
  double* s[3];
  float* s32[3];
  double* dinvS;       // 1/diag(S), pin -> 1
  float* dinvS32;
  double* dinvL;       // reference Jacobi diag_inv of the unweighted operator
  double* tlo[3];      // shifted line system: lower coefficient
  double* tdg[3];      // diagonal (later overwritten by Thomas denominators)
  double* tup[3];      // upper (later overwritten by Thomas c')
  double shift_scale;  // 2/(c_tau h_min^2)
  int ndim;
  int want_line;
};

__global__ void prep_faces_kernel(PrepArgs a) {
  const Grid3& g = a.g;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < g.ndof; idx += gridDim.x * blockDim.x) {
    int i0, i1, i2;
    coords3(g, idx, i0, i1, i2);
    const int iv[3] = {i0, i1, i2};
    const int Nv[3] = {g.N0, g.N1, g.N2};
    const int stv[3] = {g.st0, g.n2, 1};
    const double rho_i = a.rho[idx];
    double dvv[3] = {a.geo.dv[0][i0], a.geo.dv[1][i1], g.N2 > 0 ? a.geo.dv[2][i2] : 1.0};
    double diagS = 0.0, diagL = 0.0;
    for (int ax = 0; ax < 3; ++ax) {
      if (Nv[ax] == 0) continue;
      double other = 1.0;
      for (int b = 0; b < 3; ++b)
        if (b != ax) other *= dvv[b];
      double lower = 0.0, upper = 0.0, cf_lo = 0.0, cf_hi = 0.0;
      if (iv[ax] > 0) {
        double rl = a.rho[idx - stv[ax]];
        cf_lo = 2.0 / (rl + rho_i) / a.geo.dface[ax][iv[ax] - 1];
        lower = cf_lo / dvv[ax];
      }
      if (iv[ax] < Nv[ax]) {
        double rr = a.rho[idx + stv[ax]];
        cf_hi = 2.0 / (rho_i + rr) / a.geo.dface[ax][iv[ax]];
        upper = cf_hi / dvv[ax];
        double sv = cf_hi * other;
        a.s[ax][idx] = sv;
        a.s32[ax][idx] = (float)sv;
      } else {
        a.s[ax][idx] = 0.0;
        a.s32[ax][idx] = 0.0f;
      }
      diagS += cf_lo * other + cf_hi * other;
      double main = -(lower + upper);
      diagL += main;
      if (a.want_line) {
        double shift = a.shift_scale / rho_i;
        a.tlo[ax][idx] = -lower;
        a.tdg[ax][idx] = shift - main;
        a.tup[ax][idx] = -upper;
      }
    }
    if (idx == g.pin) {
      diagS = 1.0;
      diagL = 1.0;
    }
    a.dinvS[idx] = 1.0 / diagS;
    a.dinvS32[idx] = (float)(1.0 / diagS);
    a.dinvL[idx] = 1.0 / (fabs(diagL) > 1e-30 ? diagL : 1.0);
  }
}

struct LineArgs {
  int lines, n;              // number of lines, points per line
  int stride;                // element stride along the line
  int lstride_hi, lmod;      // line -> base: (l / lmod) * lstride_hi + (l % lmod) * lstride_lo
  int lstride_lo;
};

__device__ __forceinline__ int line_base(const LineArgs& L, int l) {
  return (l / L.lmod) * L.lstride_hi + (l % L.lmod) * L.lstride_lo;
}

// Thomas factors along lines: tdg -> denominators, tup -> c' (the reference's
// CPU recurrence, linalg_backend.py:496-507, with the coefficient part hoisted).
__global__ void thomas_factor_kernel(LineArgs L, const double* lo, double* dg, double* up) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L.lines) return;
  int b = line_base(L, l);
  double den = dg[b];
  double cp = (L.n > 1) ? up[b] / den : 0.0;
  up[b] = cp;
  for (int i = 1; i < L.n; ++i) {
    int e = b + i * L.stride;
    den = dg[e] - lo[e] * cp;
    dg[e] = den;
    cp = (i < L.n - 1) ? up[e] / den : 0.0;
    up[e] = cp;
  }
}

// x = T^-1 r along lines, with r[pin] read as 0.  ACC: out = (out + x) * scale.
template <bool ACC>
__global__ void thomas_solve_kernel(LineArgs L, const double* __restrict__ lo, const double* __restrict__ den,
                                    const double* __restrict__ cp, const double* __restrict__ r, double* out,
                                    double* tmp, int pin, double scale, const int* done) {
  if (done && *done) return;
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L.lines) return;
  int b = line_base(L, l);
  // forward: dp_i = (r_i - lo_i dp_{i-1}) / den_i   (stored in tmp)
  double dp = 0.0;
  for (int i = 0; i < L.n; ++i) {
    int e = b + i * L.stride;
    double ri = (e == pin) ? 0.0 : r[e];
    dp = (i == 0) ? ri / den[e] : (ri - lo[e] * dp) / den[e];
    tmp[e] = dp;
  }
  double x = 0.0;
  for (int i = L.n - 1; i >= 0; --i) {
    int e = b + i * L.stride;
    x = (i == L.n - 1) ? tmp[e] : tmp[e] - cp[e] * x;
    if (ACC) {
      double v = (out[e] + x) * scale;
      out[e] = (e == pin) ? 0.0 : v;
    } else {
      out[e] = x;
    }
  }
}

// The same exact line solve with one warp per line (the one-thread-per-line
// kernel above leaves most SMs idle and walks each line serially through
// global memory).  Lane l owns rows [l K, l K + K).  Both sweeps are affine
// recurrences, dp_i = (r_i - lo_i dp_{i-1}) / den_i and x_i = tmp_i - cp_i x_{i+1}:
// each lane composes the map of its chunk, a warp scan of the maps gives
// every lane the value entering its chunk, and the lane then runs its chunk
// with the recurrence itself (the reference's per-row arithmetic; only the
// carried-in values come from the composed maps).  tmp stays in registers.
template <bool ACC, int K>
__device__ __forceinline__ void thomas_warp_line(const LineArgs& L, const double* __restrict__ lo,
                                                 const double* __restrict__ den, const double* __restrict__ cp,
                                                 const double* __restrict__ r, double* out, int pin, double scale,
                                                 int l, int lane) {
  const int b = line_base(L, l);
  const int n = L.n;
  const int i0 = lane * K;
  // forward: compose y -> A y + B over the chunk (row 0 of the line has no carry)
  double rr[K], tmp[K];
  double A = 1.0, B = 0.0;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const int i = i0 + q;
    rr[q] = 0.0;
    if (i < n) {
      const int e = b + i * L.stride;
      const double ri = (e == pin) ? 0.0 : r[e];
      rr[q] = ri;
      const double d = den[e];
      if (i == 0) { A = 0.0; B = ri / d; }
      else {
        const double m = lo[e];
        A = -m * A / d;
        B = (ri - m * B) / d;
      }
    }
  }
  // inclusive scan of the maps across lanes (lower lanes applied first)
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const double Ap = __shfl_up_sync(0xffffffffu, A, s), Bp = __shfl_up_sync(0xffffffffu, B, s);
    if (lane >= s) { B = A * Bp + B; A = A * Ap; }
  }
  // value entering this lane's chunk = the previous lane's composed map applied to 0
  double y = __shfl_up_sync(0xffffffffu, B, 1);
  if (lane == 0) y = 0.0;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const int i = i0 + q;
    if (i < n) {
      const int e = b + i * L.stride;
      y = (i == 0) ? rr[q] / den[e] : (rr[q] - lo[e] * y) / den[e];
    }
    tmp[q] = y;
  }
  // backward: compose x -> C x + D over the chunk, from its last row down
  double C = 1.0, D = 0.0;
#pragma unroll
  for (int q = K - 1; q >= 0; --q) {
    const int i = i0 + q;
    if (i < n) {
      if (i == n - 1) { C = 0.0; D = tmp[q]; }
      else {
        const double c = cp[b + i * L.stride];
        D = tmp[q] - c * D;
        C = -c * C;
      }
    }
  }
  // suffix scan across lanes (higher lanes applied first)
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const double Cn = __shfl_down_sync(0xffffffffu, C, s), Dn = __shfl_down_sync(0xffffffffu, D, s);
    if (lane + s < 32) { D = C * Dn + D; C = C * Cn; }
  }
  double x = __shfl_down_sync(0xffffffffu, D, 1);
  if (lane == 31) x = 0.0;
#pragma unroll
  for (int q = K - 1; q >= 0; --q) {
    const int i = i0 + q;
    if (i < n) {
      const int e = b + i * L.stride;
      x = (i == n - 1) ? tmp[q] : tmp[q] - cp[e] * x;
      if (ACC) {
        const double v = (out[e] + x) * scale;
        out[e] = (e == pin) ? 0.0 : v;
      } else {
        out[e] = x;
      }
    }
  }
}

template <bool ACC, int K>
__global__ void __launch_bounds__(128) thomas_warp_kernel(LineArgs L, const double* __restrict__ lo,
                                                          const double* __restrict__ den,
                                                          const double* __restrict__ cp,
                                                          const double* __restrict__ r, double* out, int pin,
                                                          double scale, const int* done) {
  if (done && *done) return;
  const int lane = threadIdx.x & 31;
  const int l = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (l >= L.lines) return;
  thomas_warp_line<ACC, K>(L, lo, den, cp, r, out, pin, scale, l, lane);
}

// Truncated parallel cyclic reduction along lines (the reference's GPU line
// solver, linalg_backend.py:77-115): `stages` reduction steps of
//   alpha = -a_i / d_{i-s}, beta = -c_i / d_{i+s} (0 beyond the line ends),
//   a_i <- alpha a_{i-s}, c_i <- beta c_{i+s},
//   d_i <- d_i + alpha c_{i-s} + beta a_{i+s}, b_i <- b_i + alpha b_{i-s} + beta b_{i+s},
// with the stride s doubling, then x = b / d (exact when 2^stages >= n).
// One block per line; the four coefficient arrays live in shared memory,
// double-buffered.  r is read as 0 at the pin.  ACC: out = (out + x) * scale.
template <bool ACC>
__global__ void pcr_solve_kernel(LineArgs L, const double* __restrict__ lo, const double* __restrict__ dg,
                                 const double* __restrict__ up, const double* __restrict__ r, double* out, int pin,
                                 int stages, double scale, const int* done) {
  if (done && *done) return;
  extern __shared__ double sm[];
  const int n = L.n;
  double* A0 = sm;
  double* D0 = A0 + n;
  double* C0 = D0 + n;
  double* B0 = C0 + n;
  double* A1 = B0 + n;
  double* D1 = A1 + n;
  double* C1 = D1 + n;
  double* B1 = C1 + n;
  const int l = blockIdx.x;
  const int base = line_base(L, l);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int e = base + i * L.stride;
    A0[i] = lo[e];
    D0[i] = dg[e];
    C0[i] = up[e];
    B0[i] = (e == pin) ? 0.0 : r[e];
  }
  __syncthreads();
  int s = 1;
  for (int st = 0; st < stages; ++st) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double alpha = 0.0, beta = 0.0;
      double al = 0.0, cl = 0.0, bl = 0.0, ar = 0.0, cr = 0.0, br = 0.0;
      if (i >= s) {
        const double dl = D0[i - s];
        alpha = -A0[i] / (fabs(dl) > 0.0 ? dl : 1.0);
        al = A0[i - s];
        cl = C0[i - s];
        bl = B0[i - s];
      }
      if (i < n - s) {
        const double dr = D0[i + s];
        beta = -C0[i] / (fabs(dr) > 0.0 ? dr : 1.0);
        ar = A0[i + s];
        cr = C0[i + s];
        br = B0[i + s];
      }
      A1[i] = alpha * al;
      D1[i] = D0[i] + alpha * cl + beta * ar;
      C1[i] = beta * cr;
      B1[i] = B0[i] + alpha * bl + beta * br;
    }
    __syncthreads();
    double* t;
    t = A0; A0 = A1; A1 = t;
    t = D0; D0 = D1; D1 = t;
    t = C0; C0 = C1; C1 = t;
    t = B0; B0 = B1; B1 = t;
    s *= 2;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int e = base + i * L.stride;
    const double x = B0[i] / D0[i];
    if (ACC) {
      const double v = (out[e] + x) * scale;
      out[e] = (e == pin) ? 0.0 : v;
    } else {
      out[e] = x;
    }
  }
}

// ---- elementwise helpers ------------------------------------------------------

// L p (reference apply): -(S p)/W for rows != pin (pin column kept), pin row identity.
__global__ void apply_L_kernel(Grid3 g, Geo geo, const double* s0, const double* s1, const double* s2,
                               const double* __restrict__ p, double* out, const double* bsub,
                               const int* done) {
  if (done && *done) return;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < g.ndof; idx += gridDim.x * blockDim.x) {
    int i0, i1, i2;
    coords3(g, idx, i0, i1, i2);
    double v;
    if (idx == g.pin) {
      v = p[idx];
    } else {
      double d, off;
      s_row<double>(g, idx, i0, i1, i2, s0, s1, s2, [&](int j) { return p[j]; }, d, off);
      double W = geo.dv[0][i0] * geo.dv[1][i1] * (g.N2 > 0 ? geo.dv[2][i2] : 1.0);
      v = (off - d * p[idx]) / W;
    }
    out[idx] = bsub ? bsub[idx] - v : v;   // optional residual b - L p
  }
}

// weighted rhs of the CG system: b = -W rhs, b[pin] = 0; x0 from p_init (pin -> 0)
__global__ void cg_rhs_kernel(Grid3 g, Geo geo, const double* rhs, double* b, const double* p_init,
                              double* x) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < g.ndof; idx += gridDim.x * blockDim.x) {
    int i0, i1, i2;
    coords3(g, idx, i0, i1, i2);
    double W = geo.dv[0][i0] * geo.dv[1][i1] * (g.N2 > 0 ? geo.dv[2][i2] : 1.0);
    b[idx] = (idx == g.pin) ? 0.0 : -(rhs[idx] * W);
    x[idx] = (p_init && idx != g.pin) ? p_init[idx] : 0.0;
  }
}

__global__ void jacobi_L_kernel(int ndof, int pin, const double* dinvL, const double* r, double* z,
                                const int* done) {
  if (done && *done) return;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x)
    z[idx] = (idx == pin) ? 0.0 : r[idx] * dinvL[idx];
}

__global__ void copy_pin0_kernel(int ndof, int pin, const double* src, double* dst) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x)
    dst[idx] = (idx == pin) ? 0.0 : src[idx];
}

// ---- persistent PCG ----------------------------------------------------------------
//
// Chronopoulos-Gear preconditioned CG: mathematically the CG iteration SciPy's
// cg performs (stop when ||r|| < tol ||b|| at the top of an iteration), with
// the two inner products of an iteration fused into ONE grid-wide reduction:
//   gamma = (r,u), delta = (w,u), u = M r, w = S u,
//   beta = gamma/gamma_old, alpha = gamma / (delta - beta gamma / alpha_old),
//   p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s.
// The next stencil w_new = S M r_new is fused into the same pass: neighbour
// values of u_new are recomputed from (r, w, s) of the previous pass, which
// are double-buffered, so each iteration needs one barrier.

struct SolveStatus {
  long long iters;
  long long applies;
  long long refinements;   // FP64 residual replacements (mixed)
  double rr;               // final ||r||^2 of the solved system
  double bb;               // ||b||^2
  int converged;
  int pad;
};

template <typename T>
struct Cg1Vecs {
  const T* s0; const T* s1; const T* s2;   // face couplings
  const T* dinv;                           // Jacobi (1/diag S; pin -> 1)
  T* r[2]; T* w[2]; T* s[2];
  T* p;
};

struct Cg1Args {
  Grid3 g;
  Cg1Vecs<double> v64;
  Cg1Vecs<float> v32;
  const double* s64[3];    // FP64 couplings for the residual replacement (mixed)
  const double* b;         // SPD-system rhs
  double* x;               // solution (FP64 in both modes)
  long long maxiter;
  double tol;
  double replace_drop;     // mixed: replace the residual when ||r|| fell by this factor
  int x_nonzero;
  double* part;            // [2 slots][8][nblocks]
  unsigned int* count;     // monotonic arrival counter
  int* err;
  SolveStatus* st;
};

__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide sum of NV doubles through a bounded barrier on a monotonic
// arrival counter (release add / acquire poll by one thread per block); the
// partials are summed in block order by every block (identical totals).
struct GridSum {
  double* part;            // [2 slots][8][nblocks]
  unsigned int* count;     // monotonic arrival counter, zeroed before the launch
  int* err;
  unsigned int nb;         // blocks taking part (the whole grid, or one case's blocks)
  unsigned int epoch;
  unsigned int bid;        // this block's index among them

  template <int NV>
  __device__ __forceinline__ bool sum(double (&v)[NV], double* scratch) {
    tpf::block_sum<NV>(v, scratch);
    const int slot = epoch & 1;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; ++k) part[(slot * 8 + k) * nb + bid] = v[k];
      red_release_add(count, 1u);
      const unsigned int target = (epoch + 1) * nb;
      int ok = 1;
      long long spins = 0;
      while (ld_acquire(count) < target) {
        if (++spins > kSpinLimit * 8) { atomicExch(err, 1); ok = 0; break; }
        if ((spins & 1023) == 0 && *(volatile int*)err) { ok = 0; break; }
      }
      s_ok = ok;
    }
    __syncthreads();
    const bool ok = s_ok != 0;
    // every thread of the block loads partials (one L2 round trip for up to
    // blockDim.x / 32 blocks per warp), then a fixed-order reduction: warp
    // sums, then the warp totals in warp order (deterministic)
    {
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
      double acc[NV];
#pragma unroll
      for (int k = 0; k < NV; ++k) acc[k] = 0.0;
      for (unsigned int j = threadIdx.x; j < nb; j += blockDim.x) {
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(part + (slot * 8 + k) * nb + j);
      }
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        acc[k] = tpf::warp_sum(acc[k]);
        if (lane == 0) scratch[k * 16 + wid] = acc[k];
      }
      __syncthreads();
      if (threadIdx.x < NV) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += scratch[threadIdx.x * 16 + w];
        scratch[224 + threadIdx.x] = t;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = scratch[224 + k];
    __syncthreads();
    ++epoch;
    return ok;
  }
};

// r = b - S x for own nodes (x FP64, pin column zero / pin row identity)
template <typename T>
__device__ __forceinline__ void residual_pass(const Grid3& g, const double* s0, const double* s1,
                                              const double* s2, const double* b, const double* x, T* r,
                                              bool x_nonzero, double& bb, double& rr, int vb, int nvb) {
  for (NodeIter it(g, vb, nvb); it.ok(); it.next(g)) {
    const int idx = it.idx;
    double bi = b[idx];
    double ri = bi;
    if (x_nonzero) {
      double sx;
      if (idx == g.pin) sx = x[idx];
      else {
        const int i0 = it.i0, i1 = it.i1, i2 = it.i2;
        double d, off;
        s_row<double>(g, idx, i0, i1, i2, s0, s1, s2, [&](int j) { return (j == g.pin) ? 0.0 : x[j]; }, d, off);
        sx = d * x[idx] - off;
      }
      ri = bi - sx;
    }
    r[idx] = (T)ri;
    bb += bi * bi;
    rr += ri * ri;
  }
}

// u = M r, w = S u for own nodes (r read at neighbours) and the six inner
// products of the single reduction with the current search directions p, s:
// red = {(r,u), (w,u), (u,s), (p,w), (p,s), (r,r)}.  init: p = s = 0.
template <typename T>
__device__ __forceinline__ void w_pass(const Grid3& g, const Cg1Vecs<T>& v, int cur, bool init, double (&red)[6],
                                       int vb, int nvb) {
  const T* __restrict__ r = v.r[cur];
  for (NodeIter it(g, vb, nvb); it.ok(); it.next(g)) {
    const int idx = it.idx;
    const int i0 = it.i0, i1 = it.i1, i2 = it.i2;
    const T ri = r[idx];
    const T ui = v.dinv[idx] * ri;
    T wi;
    if (idx == g.pin) {
      wi = ui;
    } else {
      T d, off;
      s_row<T>(g, idx, i0, i1, i2, v.s0, v.s1, v.s2,
               [&](int j) -> T { return (j == g.pin) ? T(0) : v.dinv[j] * r[j]; }, d, off);
      wi = d * ui - off;
    }
    v.w[cur][idx] = wi;
    T si = T(0), pi = T(0);
    if (init) {
      v.s[cur][idx] = T(0);
      v.p[idx] = T(0);
    } else {
      si = v.s[cur][idx];
      pi = v.p[idx];
    }
    red[0] += (double)ri * (double)ui;
    red[1] += (double)wi * (double)ui;
    red[2] += (double)ui * (double)si;
    red[3] += (double)pi * (double)wi;
    red[4] += (double)pi * (double)si;
    red[5] += (double)ri * (double)ri;
  }
}

// The whole PCG solve of one system, run by blocks [0, nvb) of a grid (vb =
// this block's index): the full grid for a single solve, or one case's share
// of a batched launch.
template <typename T, bool MIXED>
__device__ __forceinline__ void cg1_body(const Cg1Args& a, int vb, int nvb) {
  __shared__ double scratch[256];
  GridSum gs{a.part, a.count, a.err, (unsigned int)nvb, 0u, (unsigned int)vb};
  const Grid3& g = a.g;
  const Cg1Vecs<T>& v = *reinterpret_cast<const Cg1Vecs<T>*>(MIXED ? (const void*)&a.v32 : (const void*)&a.v64);
  const int gtid = vb * blockDim.x + threadIdx.x;
  int cur = 0;
  // r0 = b - S x0
  double red0[2] = {0.0, 0.0};
  residual_pass<T>(g, a.s64[0], a.s64[1], a.s64[2], a.b, a.x, v.r[cur], a.x_nonzero != 0, red0[0], red0[1], vb, nvb);
  if (!gs.sum<2>(red0, scratch)) return;
  const double bb = red0[0];
  if (bb == 0.0) {
    for (NodeIter it(g, vb, nvb); it.ok(); it.next(g)) a.x[it.idx] = 0.0;
    if (gtid == 0) { a.st->iters = 0; a.st->applies = 0; a.st->rr = 0.0; a.st->bb = 0.0; a.st->converged = 1; }
    return;
  }
  const double atol = a.tol * sqrt(bb);
  const double atol2 = atol * atol;
  double red[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  w_pass<T>(g, v, cur, true, red, vb, nvb);
  bool ok = gs.sum<6>(red, scratch);
  // loop state: gamma_i, rr_i and the denominator (p_i, S p_i) of alpha_i
  double gamma = red[0], rr = red[5];
  double beta = 0.0, denom = red[1];
  double rr_ref = rr;            // ||r||^2 at the last FP64 residual replacement
  long long it = 0, replacements = 0, applies = a.x_nonzero ? 2 : 1;
  bool conv = false;
  while (ok) {
    const bool small = rr < atol2;
    if (small && !MIXED) { conv = true; break; }
    if (!small && it >= a.maxiter) break;
    if (MIXED && (small || rr < a.replace_drop * a.replace_drop * rr_ref)) {
      // FP64 residual replacement r = b - S x (x is FP64) followed by a CG
      // restart: in FP32 the recurrences r, s drift from b - S x and S p
      // (the true residual stalls near eps32 * kappa), so each replacement
      // starts a fresh Krylov cycle from the FP64 iterate
      double rb[2] = {0.0, 0.0};
      residual_pass<T>(g, a.s64[0], a.s64[1], a.s64[2], a.b, a.x, v.r[cur], true, rb[0], rb[1], vb, nvb);
      ++replacements;
      ++applies;
      if (!(ok = gs.sum<2>(rb, scratch))) break;
      if (rb[1] < atol2) { rr = rb[1]; conv = true; break; }
      if (it >= a.maxiter) { rr = rb[1]; break; }
      double rd[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      w_pass<T>(g, v, cur, true, rd, vb, nvb);
      ++applies;
      if (!(ok = gs.sum<6>(rd, scratch))) break;
      beta = 0.0;
      denom = rd[1];
      gamma = rd[0];
      rr = rd[5];
      rr_ref = rr;
      continue;
    }
    const double alpha_d = gamma / denom;
    const T b_t = (T)beta, alpha = (T)alpha_d;
    const int nxt = cur ^ 1;
    const T* __restrict__ rc = v.r[cur];
    const T* __restrict__ wc = v.w[cur];
    const T* __restrict__ sc = v.s[cur];
    const T* __restrict__ dinv = v.dinv;
    T* __restrict__ pv = v.p;
    double* __restrict__ xv = a.x;
    T* __restrict__ rn_out = v.r[nxt];
    T* __restrict__ sn_out = v.s[nxt];
    T* __restrict__ wn_out = v.w[nxt];
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k] = 0.0;
#pragma unroll 2
    for (NodeIter it(g, vb, nvb); it.ok(); it.next(g)) {
      const int idx = it.idx;
      const int i0 = it.i0, i1 = it.i1, i2 = it.i2;
      const T ri = rc[idx];
      const T ui = dinv[idx] * ri;
      const T si = wc[idx] + b_t * sc[idx];
      const T pi = ui + b_t * pv[idx];
      pv[idx] = pi;
      xv[idx] += alpha_d * (double)pi;
      const T rn = ri - alpha * si;
      const T un = dinv[idx] * rn;
      T wn;
      if (idx == g.pin) {
        wn = un;
      } else {
        auto unb = [&](int j) -> T {
          if (j == g.pin) return T(0);
          return dinv[j] * (rc[j] - alpha * (wc[j] + b_t * sc[j]));
        };
        T d, off;
        s_row<T>(g, idx, i0, i1, i2, v.s0, v.s1, v.s2, unb, d, off);
        wn = d * un - off;
      }
      rn_out[idx] = rn;
      sn_out[idx] = si;
      wn_out[idx] = wn;
      red[0] += (double)rn * (double)un;
      red[1] += (double)wn * (double)un;
      red[2] += (double)un * (double)si;
      red[3] += (double)pi * (double)wn;
      red[4] += (double)pi * (double)si;
      red[5] += (double)rn * (double)rn;
    }
    ok = gs.sum<6>(red, scratch);
    const double gnew = red[0];
    beta = gnew / gamma;
    denom = red[1] + beta * (red[2] + red[3]) + beta * beta * red[4];
    gamma = gnew;
    rr = red[5];
    cur = nxt;
    ++it;
    ++applies;
  }
  if (gtid == 0) {
    a.st->iters = it;
    a.st->applies = applies;
    a.st->refinements = replacements;
    a.st->rr = rr;
    a.st->bb = bb;
    a.st->converged = conv ? 1 : 0;
  }
}

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1) cg1_kernel(Cg1Args a) {
  cg1_body<T, MIXED>(a, blockIdx.x, gridDim.x);
}

// Many independent systems in one cooperative launch: case c owns blocks
// [first[c], first[c + 1]) and runs its own PCG with its own barrier counter.
constexpr int kBatchMax = 64;
struct Cg1Batch {
  Cg1Args c[kBatchMax];
  int first[kBatchMax + 1];
  int n;
};

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1) cg1_batch_kernel(const __grid_constant__ Cg1Batch b) {
  int c = 0;
  while (c + 1 < b.n && (int)blockIdx.x >= b.first[c + 1]) ++c;
  cg1_body<T, MIXED>(b.c[c], blockIdx.x - b.first[c], b.first[c + 1] - b.first[c]);
}

// ---- band-resident PCG (2-D; FP64, or FP32 under FP64 residual replacement) ----------------
//
// The same Chronopoulos-Gear iteration as cg1_body (Jacobi or none), for 2-D
// systems whose per-SM share fits in shared memory (513^2 on 148 SMs:
// ~1 780 nodes per SM in FP64, twice that in FP32).  CTA b owns the
// contiguous node range [b ndof / G, (b+1) ndof / G) (balanced to one node;
// every range is at least one row of W = n1 nodes long); its r, w, s
// (double-buffered), p, x, M^-1 and both face couplings stay in shared memory
// for the whole solve.  The stencil reaches W nodes back and forward, which
// lie in the two adjacent ranges: each CTA publishes its first and last W
// nodes' (r, w, s) before the barrier (double-buffered by iteration parity; a
// slot is rewritten only after its readers have arrived at the next barrier)
// and reads its neighbours' after it.  Per iteration: u = M r once per node
// (sub-pass 1), w = S u from shared memory (sub-pass 2), one grid-wide
// reduction; x is written back once at the end, so the only global traffic
// of an iteration is the halo and the reduction.
//
// Layout: u is stored as [W nodes before the range | the range | W nodes
// after it] and the couplings as [W nodes before | the range], so every
// neighbour is a fixed offset (+-1, +-W).  Faces on the domain boundary need
// no test: their couplings are stored as 0 (the last row's axis-0 and the
// last column's axis-1 couplings, which the previous node's axis-1 coupling
// also is at a row start) and the node values they multiply are finite
// (zero outside the domain), so they add exact zeros, as the clamped form of
// s_row does.  The pin node's u is stored as 0 (its column is zero); its own
// u is recomputed where its row needs it.
//
// MIXED (T = float): the vectors, couplings and M^-1 are FP32, x and the
// inner products FP64, and the residual is replaced by the FP64 b - S x
// (couplings from the FP64 arrays in global memory, the neighbours' x edges
// published through global memory) whenever ||r|| has fallen by
// replace_drop since the last replacement and before accepting convergence,
// followed by a CG restart -- the rule of cg1_body<float, true>.
struct BandArgs {
  Grid3 g;
  const double* s0;      // couplings to the next row (axis 0), 0 on the last row
  const double* s1;      // couplings to the next column (axis 1), 0 on the last column
  const double* dinv;    // Jacobi 1/diag(S) (pin -> 1), or ones
  const float* s0f;      // FP32 copies (MIXED)
  const float* s1f;
  const float* dinvf;
  const double* b;       // SPD-system rhs
  double* x;             // solution
  long long maxiter;
  double tol;
  double replace_drop;   // MIXED: replace the residual when ||r|| fell by this factor
  int x_nonzero;
  int n_max;             // nodes of the largest range
  void* pub;             // [2 parity][G][2 side: first / last W nodes][3 vec: r, w, s][W] of T
  double* part;          // [2 slots][8][G]
  unsigned int* count;   // monotonic arrival counter
  int* err;
  SolveStatus* st;
};

// shared-memory bytes: x (FP64) + 11 range arrays of T + 6 rows of halo of T
// (u 2, couplings 2, M^-1 2)
template <typename T>
inline size_t band_smem_bytes(int n_max, int n1) {
  return (size_t)n_max * sizeof(double) + ((size_t)11 * n_max + 6 * (size_t)n1) * sizeof(T);
}

// The whole band-resident solve of one system by blocks [0, G) of a grid
// (bid = this block's index): the full grid for a single solve, or one
// case's share of a batched launch.
template <typename T, bool MIXED>
__device__ __forceinline__ void cg1_band_body(const BandArgs& a, const int bid, const int G) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double scratch[256];
  const Grid3& g = a.g;
  const int t = threadIdx.x, NT = blockDim.x;
  const int W = g.n1, NM = a.n_max;
  const int base = (int)((long long)bid * g.ndof / G), end = (int)((long long)(bid + 1) * g.ndof / G);
  const int nown = end - base;
  double* X = reinterpret_cast<double*>(smraw);
  T* sm = reinterpret_cast<T*>(smraw + (size_t)NM * sizeof(double));
  T* rb[2] = {sm, sm + NM};
  T* wb[2] = {sm + 2 * NM, sm + 3 * NM};
  T* sb[2] = {sm + 4 * NM, sm + 5 * NM};
  T* P = sm + 6 * NM;
  T* D = sm + 7 * NM;
  T* Ue = sm + 8 * NM;            // [W before | range | W after]  (NM + 2 W)
  T* A0e = Ue + NM + 2 * W;       // [W before | range]            (NM + W)
  T* A1e = A0e + NM + W;          // [W before | range]            (NM + W)
  T* HD = A1e + NM + W;           // [2][W]: M^-1 of the nodes before / after the range
  T* Ua = Ue + W + nown;          // u of the W nodes after the range
  const T* s0t;
  const T* s1t;
  const T* dit;
  if constexpr (MIXED) {
    s0t = a.s0f; s1t = a.s1f; dit = a.dinvf;
  } else {
    s0t = a.s0; s1t = a.s1; dit = a.dinv;
  }
  T* const pubv = static_cast<T*>(a.pub);
  const bool has_up = bid > 0, has_dn = bid < G - 1;
  GridSum gs{a.part, a.count, a.err, (unsigned int)G, 0u, (unsigned int)bid};
  auto pub = [&](int par, int blk, int side, int vec) -> T* {
    return pubv + ((((size_t)par * G + blk) * 2 + side) * 3 + vec) * W;
  };
  // S-row of own node o on a field V stored in the extended layout
  auto stencil = [&](const T* V, int o, T& d, T& off) {
    const T sm0 = A0e[o], sp0 = A0e[o + W], sm1 = A1e[o + W - 1], sp1 = A1e[o + W];
    d = (sm0 + sp0) + (sm1 + sp1);
    off = sm0 * V[o] + sp0 * V[o + 2 * W] + sm1 * V[o + W - 1] + sp1 * V[o + W + 1];
  };
  // global index of halo entry k of side 0 (the W nodes before) / 1 (after)
  auto hq = [&](int side, int k) { return side == 0 ? base - W + k : end + k; };
  auto hlive = [&](int side, int k) {
    const int q = hq(side, k);
    return (side == 0 ? has_up : has_dn) && q >= 0 && q < g.ndof;
  };
  auto hslot = [&](int side, int k) -> T& { return side == 0 ? Ue[k] : Ua[k]; };
  // FP64 (S x)_idx of own node o (MIXED): x of own nodes from shared memory,
  // of the neighbour ranges' edges from global memory, couplings FP64 from
  // global memory (0 on boundary faces; out-of-domain neighbours skipped)
  auto sx64 = [&](int o) -> double {
    const int idx = base + o;
    if (idx == g.pin) return X[o];
    auto xv = [&](int q) -> double {
      if (q == g.pin) return 0.0;
      const int oo = q - base;
      return (oo >= 0 && oo < nown) ? X[oo] : __ldcg(a.x + q);
    };
    const double sm0 = idx >= W ? a.s0[idx - W] : 0.0, sp0 = a.s0[idx];
    const double sm1 = idx >= 1 ? a.s1[idx - 1] : 0.0, sp1 = a.s1[idx];
    const double d = (sm0 + sp0) + (sm1 + sp1);
    const double off = (idx >= W ? sm0 * xv(idx - W) : 0.0) + (idx + W < g.ndof ? sp0 * xv(idx + W) : 0.0) +
                       (idx >= 1 ? sm1 * xv(idx - 1) : 0.0) + (idx + 1 < g.ndof ? sp1 * xv(idx + 1) : 0.0);
    return d * X[o] - off;
  };
  // u = M r, w = S u and the six inner products with p = s = 0, r in rb[c]
  // and its halo published at parity c ^ 1; (r, w, s = 0) edges published at
  // parity c
  auto init_pass = [&](int c, double (&red)[6]) {
    for (int k = t; k < 2 * W; k += NT) {
      const int side = k / W, kk = k - side * W;
      T u = T(0);
      if (hlive(side, kk) && hq(side, kk) != g.pin)
        u = HD[k] * __ldcg(pub(c ^ 1, side == 0 ? bid - 1 : bid + 1, side ^ 1, 0) + kk);
      hslot(side, kk) = u;
    }
    for (int o = t; o < nown; o += NT) Ue[W + o] = (base + o == g.pin) ? T(0) : D[o] * rb[c][o];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k] = 0.0;
    for (int o = t; o < nown; o += NT) {
      const int idx = base + o;
      const T ri = rb[c][o];
      T ui, wi;
      if (idx == g.pin) {
        ui = D[o] * ri;
        wi = ui;
      } else {
        ui = Ue[W + o];
        T d, off;
        stencil(Ue, o, d, off);
        wi = d * ui - off;
      }
      wb[c][o] = wi;
      sb[c][o] = T(0);
      P[o] = T(0);
      red[0] += (double)ri * (double)ui;
      red[1] += (double)wi * (double)ui;
      red[5] += (double)ri * (double)ri;
      if (o < W) { pub(c, bid, 0, 0)[o] = ri; pub(c, bid, 0, 1)[o] = wi; pub(c, bid, 0, 2)[o] = T(0); }
      if (o >= nown - W) {
        const int k = o - (nown - W);
        pub(c, bid, 1, 0)[k] = ri; pub(c, bid, 1, 1)[k] = wi; pub(c, bid, 1, 2)[k] = T(0);
      }
    }
  };

  // static data
  for (int o = t; o < nown; o += NT) {
    D[o] = dit[base + o];
    A0e[W + o] = s0t[base + o];
    A1e[W + o] = s1t[base + o];
    X[o] = a.x[base + o];
  }
  for (int k = t; k < 2 * W; k += NT) {
    const int side = k / W, kk = k - side * W;
    const bool live = hlive(side, kk);
    HD[k] = live ? dit[hq(side, kk)] : T(0);
    if (side == 0) {
      A0e[kk] = live ? s0t[hq(0, kk)] : T(0);
      A1e[kk] = live ? s1t[hq(0, kk)] : T(0);
    }
  }
  __syncthreads();

  // r0 = b - S x (pin column zero / pin row identity); FP64: x, pin zeroed,
  // staged in Ue; MIXED: sx64 over the initial x in global memory
  double red0[2] = {0.0, 0.0};
  if (!MIXED && a.x_nonzero) {
    for (int o = t; o < nown; o += NT) Ue[W + o] = (base + o == g.pin) ? T(0) : (T)X[o];
    for (int k = t; k < 2 * W; k += NT) {
      const int side = k / W, kk = k - side * W;
      const int q = hq(side, kk);
      hslot(side, kk) = (hlive(side, kk) && q != g.pin) ? (T)a.x[q] : T(0);
    }
    __syncthreads();
  }
  for (int o = t; o < nown; o += NT) {
    const int idx = base + o;
    const double bi = a.b[idx];
    double ri = bi;
    if (a.x_nonzero) {
      double sx;
      if constexpr (MIXED) {
        sx = sx64(o);
      } else {
        if (idx == g.pin) {
          sx = X[o];
        } else {
          T d, off;
          stencil(Ue, o, d, off);
          sx = d * X[o] - off;
        }
      }
      ri = bi - sx;
    }
    rb[0][o] = (T)ri;
    red0[0] += bi * bi;
    red0[1] += ri * ri;
    if (o < W) pub(1, bid, 0, 0)[o] = (T)ri;
    if (o >= nown - W) pub(1, bid, 1, 0)[o - (nown - W)] = (T)ri;
  }
  if (!gs.sum<2>(red0, scratch)) return;
  const double bb = red0[0];
  if (bb == 0.0) {
    for (int o = t; o < nown; o += NT) a.x[base + o] = 0.0;
    if (bid == 0 && t == 0) {
      a.st->iters = 0; a.st->applies = 0; a.st->refinements = 0; a.st->rr = 0.0; a.st->bb = 0.0;
      a.st->converged = 1;
    }
    return;
  }
  const double atol = a.tol * sqrt(bb);
  const double atol2 = atol * atol;

  double red[6];
  init_pass(0, red);
  bool ok = gs.sum<6>(red, scratch);
  double gamma = red[0], rr = red[5];
  double beta = 0.0, denom = red[1];
  double rr_ref = rr;    // ||r||^2 at the last FP64 residual replacement (MIXED)
  long long it = 0, replacements = 0, applies = a.x_nonzero ? 2 : 1;
  bool conv = false;
  int cur = 0;
  constexpr int KH = 3;   // halo entries per thread: 2 * W <= KH * kThreads
  while (ok) {
    if constexpr (MIXED) {
      const bool small = rr < atol2;
      if (!small && it >= a.maxiter) break;
      if (small || rr < a.replace_drop * a.replace_drop * rr_ref) {
        // publish the x edges, barrier, r = b - S x in FP64 (halo r at
        // parity cur ^ 1), barrier with ||r||^2, then a CG restart
        for (int o = t; o < nown; o += NT)
          if (o < W || o >= nown - W) a.x[base + o] = X[o];
        double bar1[1] = {0.0};
        if (!(ok = gs.sum<1>(bar1, scratch))) break;
        double rt[1] = {0.0};
        for (int o = t; o < nown; o += NT) {
          const double ri = a.b[base + o] - sx64(o);
          rb[cur][o] = (T)ri;
          rt[0] += ri * ri;
          if (o < W) pub(cur ^ 1, bid, 0, 0)[o] = (T)ri;
          if (o >= nown - W) pub(cur ^ 1, bid, 1, 0)[o - (nown - W)] = (T)ri;
        }
        ++replacements;
        ++applies;
        if (!(ok = gs.sum<1>(rt, scratch))) break;
        if (rt[0] < atol2) { rr = rt[0]; conv = true; break; }
        if (it >= a.maxiter) { rr = rt[0]; break; }
        init_pass(cur, red);
        ++applies;
        if (!(ok = gs.sum<6>(red, scratch))) break;
        beta = 0.0;
        denom = red[1];
        gamma = red[0];
        rr = red[5];
        rr_ref = rr;
        continue;
      }
    } else {
      if (rr < atol2) { conv = true; break; }
      if (it >= a.maxiter) break;
    }
    const double alpha_d = gamma / denom;
    const T alpha = (T)alpha_d, bt = (T)beta;
    const int nxt = cur ^ 1;
    // halo (r, w, s) of the neighbour ranges: loads in flight during sub-pass 1
    T hr[KH], hw[KH], hs[KH];
#pragma unroll
    for (int e = 0; e < KH; ++e) {
      const int k = t + e * NT;
      hr[e] = hw[e] = hs[e] = T(0);
      if (k < 2 * W) {
        const int side = k / W, kk = k - side * W;
        if (hlive(side, kk)) {
          const int nb = side == 0 ? bid - 1 : bid + 1;
          hr[e] = __ldcg(pub(cur, nb, side ^ 1, 0) + kk);
          hw[e] = __ldcg(pub(cur, nb, side ^ 1, 1) + kk);
          hs[e] = __ldcg(pub(cur, nb, side ^ 1, 2) + kk);
        }
      }
    }
    // sub-pass 1: p, x, r, s and u = M r_new for own nodes
    const T* __restrict__ rc = rb[cur];
    const T* __restrict__ wc = wb[cur];
    const T* __restrict__ sc = sb[cur];
    T* __restrict__ rn_o = rb[nxt];
    T* __restrict__ sn_o = sb[nxt];
    for (int o = t; o < nown; o += NT) {
      const T ri = rc[o];
      const T ui = D[o] * ri;
      const T si = wc[o] + bt * sc[o];
      const T pi = ui + bt * P[o];
      P[o] = pi;
      X[o] += alpha_d * (double)pi;
      const T rn = ri - alpha * si;
      rn_o[o] = rn;
      sn_o[o] = si;
      Ue[W + o] = (base + o == g.pin) ? T(0) : D[o] * rn;
    }
#pragma unroll
    for (int e = 0; e < KH; ++e) {
      const int k = t + e * NT;
      if (k < 2 * W) {
        const int side = k / W, kk = k - side * W;
        hslot(side, kk) =
            (!hlive(side, kk) || hq(side, kk) == g.pin) ? T(0) : HD[k] * (hr[e] - alpha * (hw[e] + bt * hs[e]));
      }
    }
    __syncthreads();
    // sub-pass 2: w = S u, the six inner products, publication of the edges
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k] = 0.0;
    T* __restrict__ wn_o = wb[nxt];
    for (int o = t; o < nown; o += NT) {
      const T rn = rn_o[o], si = sn_o[o], pi = P[o];
      T un, wn;
      if (base + o == g.pin) {
        un = D[o] * rn;
        wn = un;
      } else {
        un = Ue[W + o];
        T d, off;
        stencil(Ue, o, d, off);
        wn = d * un - off;
      }
      wn_o[o] = wn;
      red[0] += (double)rn * (double)un;
      red[1] += (double)wn * (double)un;
      red[2] += (double)un * (double)si;
      red[3] += (double)pi * (double)wn;
      red[4] += (double)pi * (double)si;
      red[5] += (double)rn * (double)rn;
      if (o < W) { pub(nxt, bid, 0, 0)[o] = rn; pub(nxt, bid, 0, 1)[o] = wn; pub(nxt, bid, 0, 2)[o] = si; }
      if (o >= nown - W) {
        const int k = o - (nown - W);
        pub(nxt, bid, 1, 0)[k] = rn; pub(nxt, bid, 1, 1)[k] = wn; pub(nxt, bid, 1, 2)[k] = si;
      }
    }
    ok = gs.sum<6>(red, scratch);
    const double gnew = red[0];
    beta = gnew / gamma;
    denom = red[1] + beta * (red[2] + red[3]) + beta * beta * red[4];
    gamma = gnew;
    rr = red[5];
    cur = nxt;
    ++it;
    ++applies;
  }
  for (int o = t; o < nown; o += NT) a.x[base + o] = X[o];
  if (bid == 0 && t == 0) {
    a.st->iters = it;
    a.st->applies = applies;
    a.st->refinements = replacements;
    a.st->rr = rr;
    a.st->bb = bb;
    a.st->converged = conv ? 1 : 0;
  }
}

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1) cg1_band_kernel(BandArgs a) {
  cg1_band_body<T, MIXED>(a, blockIdx.x, gridDim.x);
}

// Many independent 2-D systems in one cooperative launch, each band-resident
// in the shared memory of its own blocks: case c owns blocks [first[c],
// first[c + 1]) with its own barrier counter, halo buffer and status.
struct BandBatch {
  BandArgs c[kBatchMax];
  int first[kBatchMax + 1];
  int n;
};

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1) cg1_band_batch_kernel(const __grid_constant__ BandBatch b) {
  int c = 0;
  while (c + 1 < b.n && (int)blockIdx.x >= b.first[c + 1]) ++c;
  cg1_band_body<T, MIXED>(b.c[c], blockIdx.x - b.first[c], b.first[c + 1] - b.first[c]);
}

}  // namespace

namespace {

// ---- streaming PCG (large systems) --------------------------------------------------
//
// The same Jacobi-PCG recurrences as cg1_kernel (Chronopoulos-Gear, one
// reduction per iteration, SciPy's stopping rule), for systems whose vectors
// stream from HBM (3-D grids): an iteration is two ordinary kernels at full
// occupancy instead of one persistent kernel with one CTA per SM, since the
// persistent kernel's register budget (126 per thread) leaves 16 warps per SM,
// too few loads in flight to stream at HBM bandwidth.
//   update : s = w + beta s, p = M r + beta p, x += alpha p, r -= alpha s
//   stencil: w = S M r (M r recomputed at the neighbours), the six inner
//            products; the last block to finish sums the block partials in
//            block order and advances the scalars (alpha, beta, ...) and the
//            convergence state on the device.
// Chunks of iterations are captured as one CUDA graph and replayed; every
// kernel returns at once after the device-side state says done, so the host
// reads the state once per chunk.

struct CgScal {
  double gamma, denom, beta, rr, bb, atol2, tol, pad;
  long long it, applies, maxiter, pad2;
  int done, conv, x_nonzero;
  unsigned int arrive;
};

__device__ __forceinline__ bool cgs_last_block(CgScal* sc) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int prev = atomicAdd(&sc->arrive, 1u);
    s_last = (prev == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last != 0;
}

// sum of NV block partials part[k * nb + b] in block order (same tree every call)
template <int NV>
__device__ __forceinline__ void cgs_sum_partials(const double* part, int nb, double (&v)[NV], double* scratch) {
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += __ldcg(part + (size_t)k * nb + b);
  }
  tpf::block_sum<NV>(v, scratch);
}

// r = b - S x (x_nonzero) or b; then (b, b), (r, r)
__global__ void __launch_bounds__(256) cgs_resid_kernel(Grid3 g, const double* s0, const double* s1,
                                                        const double* s2, const double* b, const double* x,
                                                        double* r, double* part, CgScal* sc) {
  __shared__ double scratch[2 * 32];
  double v[2] = {0.0, 0.0};
  const bool xnz = sc->x_nonzero != 0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < g.ndof; idx += gridDim.x * blockDim.x) {
    const double bi = b[idx];
    double ri = bi;
    if (xnz) {
      double sx;
      if (idx == g.pin) sx = x[idx];
      else {
        int i0, i1, i2;
        coords3(g, idx, i0, i1, i2);
        double d, off;
        s_row<double>(g, idx, i0, i1, i2, s0, s1, s2, [&](int j) { return (j == g.pin) ? 0.0 : x[j]; }, d, off);
        sx = d * x[idx] - off;
      }
      ri = bi - sx;
    }
    r[idx] = ri;
    v[0] += bi * bi;
    v[1] += ri * ri;
  }
  tpf::block_sum<2>(v, scratch);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v[0];
    part[gridDim.x + blockIdx.x] = v[1];
  }
  if (!cgs_last_block(sc)) return;
  double t[2];
  cgs_sum_partials<2>(part, gridDim.x, t, scratch);
  if (threadIdx.x == 0) {
    sc->arrive = 0u;
    sc->bb = t[0];
    sc->rr = t[1];
    const double atol = sc->tol * sqrt(t[0]);
    sc->atol2 = atol * atol;
    sc->it = 0;
    sc->applies = 0;
    sc->conv = 0;
    sc->done = 0;
    if (t[0] == 0.0) { sc->done = 1; sc->conv = 1; }
  }
}

// Inner products of an iteration: {(r,u), (w,u), (u,s), (p,w), (p,s), (r,r)}
// with the new r, u = M r, s, p and w = S u.  The update kernel sums the four
// without w (slots 0, 2, 4, 5 of part), the stencil kernel the two with w
// (slots 1, 3); the stencil kernel's last block adds them up.

// INIT: u = M r, s = p = 0.  Else: s = w + beta s, p = M r + beta p,
// x += alpha p, r -= alpha s, u = M r (new r).
template <bool INIT>
__device__ __forceinline__ void cgs_update_node(int idx, int pin, double ri, double di, double wi, double svi,
                                                double pvi, double& xi, double alpha, double beta, double& rn,
                                                double& si, double& pi, double& un) {
  rn = ri;
  si = 0.0;
  pi = 0.0;
  if (!INIT) {
    si = wi + beta * svi;
    pi = di * ri + beta * pvi;
    xi += alpha * pi;
    rn = ri - alpha * si;
  }
  un = (idx == pin) ? 0.0 : di * rn;   // r[pin] stays 0: u[pin] = 0 either way
}

// Two consecutive nodes per thread and trip (16-byte loads and stores; the
// vectors come from cudaMalloc, so even node indices are 16-byte aligned).
// (bid, nblk: this block's index among the nblk blocks working on the system)
template <bool INIT>
__device__ __forceinline__ void cgs_update_body(int bid, int nblk, int ndof, int pin, const double* __restrict__ dinv,
                                                const double* __restrict__ w, double* __restrict__ sv,
                                                double* __restrict__ pv, double* __restrict__ x,
                                                double* __restrict__ r, double* __restrict__ u, double* part,
                                                const CgScal* sc) {
  if (sc->done) return;
  __shared__ double scratch[4 * 32];
  double alpha = 0.0, beta = 0.0;
  if (!INIT) {
    alpha = sc->gamma / sc->denom;
    beta = sc->beta;
  }
  double red[4] = {0.0, 0.0, 0.0, 0.0};
  const int npair = ndof >> 1;
  for (int k = bid * blockDim.x + threadIdx.x; k < npair; k += nblk * blockDim.x) {
    const int i0 = 2 * k;
    const double2 r2 = reinterpret_cast<const double2*>(r)[k];
    const double2 d2 = reinterpret_cast<const double2*>(dinv)[k];
    double2 w2 = make_double2(0.0, 0.0), s2 = w2, p2 = w2, x2 = w2;
    if (!INIT) {
      w2 = reinterpret_cast<const double2*>(w)[k];
      s2 = reinterpret_cast<const double2*>(sv)[k];
      p2 = reinterpret_cast<const double2*>(pv)[k];
      x2 = reinterpret_cast<const double2*>(x)[k];
    }
    double rn0, si0, pi0, un0, rn1, si1, pi1, un1;
    cgs_update_node<INIT>(i0, pin, r2.x, d2.x, w2.x, s2.x, p2.x, x2.x, alpha, beta, rn0, si0, pi0, un0);
    cgs_update_node<INIT>(i0 + 1, pin, r2.y, d2.y, w2.y, s2.y, p2.y, x2.y, alpha, beta, rn1, si1, pi1, un1);
    if (!INIT) {
      reinterpret_cast<double2*>(x)[k] = x2;
      reinterpret_cast<double2*>(r)[k] = make_double2(rn0, rn1);
    }
    reinterpret_cast<double2*>(sv)[k] = make_double2(si0, si1);
    reinterpret_cast<double2*>(pv)[k] = make_double2(pi0, pi1);
    reinterpret_cast<double2*>(u)[k] = make_double2(un0, un1);
    red[0] += rn0 * un0;
    red[1] += un0 * si0;
    red[2] += pi0 * si0;
    red[3] += rn0 * rn0;
    red[0] += rn1 * un1;
    red[1] += un1 * si1;
    red[2] += pi1 * si1;
    red[3] += rn1 * rn1;
  }
  if ((ndof & 1) && bid == nblk - 1 && threadIdx.x == 0) {   // odd node count: the last node
    const int i = ndof - 1;
    double xi = INIT ? 0.0 : x[i];
    double rn, si, pi, un;
    cgs_update_node<INIT>(i, pin, r[i], dinv[i], INIT ? 0.0 : w[i], INIT ? 0.0 : sv[i], INIT ? 0.0 : pv[i], xi,
                          alpha, beta, rn, si, pi, un);
    if (!INIT) {
      x[i] = xi;
      r[i] = rn;
    }
    sv[i] = si;
    pv[i] = pi;
    u[i] = un;
    red[0] += rn * un;
    red[1] += un * si;
    red[2] += pi * si;
    red[3] += rn * rn;
  }
  tpf::block_sum<4>(red, scratch);
  if (threadIdx.x == 0) {
    part[(size_t)0 * nblk + bid] = red[0];
    part[(size_t)2 * nblk + bid] = red[1];
    part[(size_t)4 * nblk + bid] = red[2];
    part[(size_t)5 * nblk + bid] = red[3];
  }
}

template <bool INIT>
__global__ void __launch_bounds__(256) cgs_update_kernel(int ndof, int pin, const double* __restrict__ dinv,
                                                         const double* __restrict__ w, double* __restrict__ sv,
                                                         double* __restrict__ pv, double* __restrict__ x,
                                                         double* __restrict__ r, double* __restrict__ u,
                                                         double* part, const CgScal* sc) {
  cgs_update_body<INIT>(blockIdx.x, gridDim.x, ndof, pin, dinv, w, sv, pv, x, r, u, part, sc);
}

// w = S u, marching along axis 0: thread j owns column j of the (axis 1,
// axis 2) plane for planes [c0, c1) of chunk blockIdx.y and keeps u and the
// axis-0 coupling of the planes below / above in registers, so u is read
// from HBM once; the pin row is the identity (w = u).  Then (w, u), (p, w);
// the last block to finish advances the scalars.  Same grid for every launch
// (the partial sums are indexed by the flattened block id).
// (bx, by: this block's column tile and plane chunk in the system's gx x gy grid)
template <bool INIT>
__device__ __forceinline__ void cgs_stencil_body(int bx, int by, int gx, int gy, const Grid3& g, int chunk,
                                                 const double* __restrict__ s0, const double* __restrict__ s1,
                                                 const double* __restrict__ s2, const double* __restrict__ u,
                                                 const double* __restrict__ pv, double* __restrict__ w, double* part,
                                                 CgScal* sc) {
  if (sc->done) return;
  __shared__ double scratch[6 * 32];
  const int nplane = g.st0;
  const int j = bx * blockDim.x + threadIdx.x;
  const int c0 = by * chunk;
  const int c1 = min(c0 + chunk, g.n0);
  double red[2] = {0.0, 0.0};
  if (j < nplane && c0 < c1) {
    const bool three = g.N2 > 0;
    const int i1 = three ? j / g.n2 : j;
    const int i2 = three ? j - i1 * g.n2 : 0;
    // in-plane neighbours (clamped to the node itself on the walls, whose
    // couplings are stored zeros or masked)
    const int a1 = three ? g.n2 : 1;
    const bool lo1 = i1 > 0, hi1 = i1 < g.N1;
    const bool lo2 = three && i2 > 0, hi2 = three && i2 < g.N2;
    int idx = c0 * nplane + j;
    double um = (c0 > 0) ? u[idx - nplane] : 0.0;
    double s0m = (c0 > 0) ? s0[idx - nplane] : 0.0;
    double uc = u[idx];
#pragma unroll 4
    for (int i0 = c0; i0 < c1; ++i0, idx += nplane) {
      const double up = (i0 < g.N0) ? u[idx + nplane] : 0.0;
      const double s0p = s0[idx];   // zero on the last plane
      const double s1m = lo1 ? s1[idx - a1] : 0.0, s1p = s1[idx];
      double d = (s0m + s0p) + (s1m + s1p);
      double acc = s0m * um + s0p * up + s1m * (lo1 ? u[idx - a1] : 0.0) + s1p * (hi1 ? u[idx + a1] : 0.0);
      if (three) {
        const double s2m = lo2 ? s2[idx - 1] : 0.0, s2p = s2[idx];
        d += s2m + s2p;
        acc += s2m * (lo2 ? u[idx - 1] : 0.0) + s2p * (hi2 ? u[idx + 1] : 0.0);
      }
      const double wi = (idx == g.pin) ? uc : d * uc - acc;
      w[idx] = wi;
      red[0] += wi * uc;
      red[1] += pv[idx] * wi;
      um = uc;
      uc = up;
      s0m = s0p;
    }
  }
  tpf::block_sum<2>(red, scratch);
  const int nb = gx * gy;
  const int bid = by * gx + bx;
  if (threadIdx.x == 0) {
    part[(size_t)1 * nb + bid] = red[0];
    part[(size_t)3 * nb + bid] = red[1];
  }
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&sc->arrive, 1u) == (unsigned int)nb - 1) ? 1 : 0;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double t[6];
  cgs_sum_partials<6>(part, nb, t, scratch);
  if (threadIdx.x == 0) {
    sc->arrive = 0u;
    if (INIT) {
      sc->gamma = t[0];
      sc->denom = t[1];
      sc->beta = 0.0;
      sc->applies = sc->x_nonzero ? 2 : 1;
    } else {
      const double gnew = t[0];
      const double beta = gnew / sc->gamma;
      sc->beta = beta;
      sc->denom = t[1] + beta * (t[2] + t[3]) + beta * beta * t[4];
      sc->gamma = gnew;
      sc->it += 1;
      sc->applies += 1;
    }
    sc->rr = t[5];
    if (t[5] < sc->atol2) { sc->conv = 1; sc->done = 1; }
    else if (sc->it >= sc->maxiter) sc->done = 1;
  }
}

template <bool INIT>
__global__ void __launch_bounds__(256) cgs_stencil_kernel(Grid3 g, int chunk, const double* __restrict__ s0,
                                                          const double* __restrict__ s1,
                                                          const double* __restrict__ s2,
                                                          const double* __restrict__ u, const double* __restrict__ pv,
                                                          double* __restrict__ w, double* part, CgScal* sc) {
  cgs_stencil_body<INIT>(blockIdx.x, blockIdx.y, gridDim.x, gridDim.y, g, chunk, s0, s1, s2, u, pv, w, part, sc);
}

// ---- batched streaming PCG: many systems' iterations in the same two launches ----
// Each system keeps its own vectors, partial sums and scalars (its own last
// block advances them); system c owns the blocks [first[c], first[c + 1]) of
// both launches (gx[c] x gy[c] of them, the same count for the update), and
// its blocks return at once after its solve is done.
struct CgsSys {
  Grid3 g;
  int chunk, gx, gy;
  const double *s0, *s1, *s2, *dinv;
  double *x, *r, *u, *w, *sv, *pv, *part;
  CgScal* sc;
};
struct CgsBatch {
  CgsSys c[kBatchMax];
  int first[kBatchMax + 1];
  int n;
};

__device__ __forceinline__ int cgs_batch_system(const CgsBatch& b, int blk) {
  int lo = 0, hi = b.n - 1;   // the system whose block range holds blk
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (blk >= b.first[mid]) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(256) cgsb_update_kernel(const __grid_constant__ CgsBatch b) {
  const int c = cgs_batch_system(b, blockIdx.x);
  const CgsSys& y = b.c[c];
  cgs_update_body<false>(blockIdx.x - b.first[c], b.first[c + 1] - b.first[c], y.g.ndof, y.g.pin, y.dinv, y.w,
                         y.sv, y.pv, y.x, y.r, y.u, y.part, y.sc);
}

__global__ void __launch_bounds__(256) cgsb_stencil_kernel(const __grid_constant__ CgsBatch b) {
  const int c = cgs_batch_system(b, blockIdx.x);
  const CgsSys& y = b.c[c];
  const int lid = blockIdx.x - b.first[c];
  cgs_stencil_body<false>(lid % y.gx, lid / y.gx, y.gx, y.gy, y.g, y.chunk, y.s0, y.s1, y.s2, y.u, y.pv, y.w,
                          y.part, y.sc);
}

// number of systems still iterating
__global__ void cgsb_pending_kernel(const __grid_constant__ CgsBatch b, int* pending) {
  int k = 0;
  for (int c = threadIdx.x; c < b.n; c += blockDim.x) k += b.c[c].sc->done ? 0 : 1;
  k = tpf::warp_sum(k);
  if (threadIdx.x == 0) *pending = k;
}

__global__ void cgs_init_kernel(CgScal* sc, double tol, long long maxiter, int x_nonzero) {
  CgScal z{};
  z.tol = tol;
  z.maxiter = maxiter;
  z.x_nonzero = x_nonzero;
  *sc = z;
}

// body of the captured while node: run again while the solve is not done
__global__ void cgs_cond_kernel(const CgScal* sc, cudaGraphConditionalHandle handle) {
  cudaGraphSetConditional(handle, sc->done ? 0u : 1u);
}

// p = x with p[pin] = 0 (x = 0 when the right-hand side is zero)
__global__ void cgs_finish_kernel(int ndof, int pin, const CgScal* sc, const double* __restrict__ x,
                                  double* __restrict__ p) {
  const bool zero = sc->bb == 0.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x)
    p[idx] = (zero || idx == pin) ? 0.0 : x[idx];
}

}  // namespace

// ---- handle -------------------------------------------------------------------------

struct tpf_ppe {
  int ndim = 2;
  Grid3 g{};
  tpf_ppe_options o{};
  double h_min = 0.0;
  std::vector<std::vector<double>> coords;
  // geometry
  double* dv[3] = {nullptr, nullptr, nullptr};
  double* dface[3] = {nullptr, nullptr, nullptr};
  // operator state
  double* s[3] = {nullptr, nullptr, nullptr};
  float* s32[3] = {nullptr, nullptr, nullptr};
  double* dinvS = nullptr;
  float* dinvS32 = nullptr;
  double* dinvL = nullptr;
  double* tlo[3] = {nullptr, nullptr, nullptr};
  double* tden[3] = {nullptr, nullptr, nullptr};
  double* tcp[3] = {nullptr, nullptr, nullptr};
  bool prepared = false;
  int line_ready = 0;   // line-preconditioner state of the last prepare (0 none, else the precond kind)
  // Krylov workspace
  double* x = nullptr; double* r = nullptr; double* z = nullptr; double* p0 = nullptr; double* p1 = nullptr;
  double* q = nullptr; double* b = nullptr; double* t1 = nullptr; double* t2 = nullptr;
  double* c64[7] = {};            // CG: r[2], w[2], s[2], p (FP64)
  float* c32[7] = {};             // CG: r[2], w[2], s[2], p (FP32, mixed)
  double* ones64 = nullptr;
  float* ones32 = nullptr;
  double* V = nullptr;            // GMRES basis (restart+1) x ndof
  int V_cols = 0;
  double* gm = nullptr;           // H | givens | S | y | hcol | hcol2 | norm
  GmState* gst = nullptr;
  double* part = nullptr;
  int part_len = 0;
  unsigned int* bar = nullptr;
  int* err = nullptr;
  cudaGraphExec_t gm_exec = nullptr;   // one GMRES restart cycle, captured
  cudaGraphExec_t cg_exec = nullptr;   // a chunk of streaming-PCG iterations, captured
  long long cg_key[6] = {};
  void* cgs = nullptr;                 // streaming-PCG device scalars (CgScal)
  int* batch_pending = nullptr;        // systems still iterating in a batched streaming solve
  int pending = 0;                     // captured CG solve: 1 status in st, 2 in cgs
  cudaStream_t cap = nullptr;          // stream the cycle is captured on (never the caller's)
  long long gm_key[6] = {};
  double* band_pub = nullptr;     // halo rows of the band-resident PCG
  size_t band_pub_len = 0;
  int cg_kernel = 0;              // 0 auto, 1 global-memory persistent PCG, 2 band-resident PCG
  SolveStatus* st = nullptr;
  int coop_blocks = 0;
  int ew_blocks = 0;
  std::vector<void*> allocs;
};

namespace {

template <typename T>
int dalloc(tpf_ppe* h, T** p, size_t n) {
  if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    tpf::set_error("cudaMalloc of %zu bytes failed", n * sizeof(T));
    return TPF_ECUDA;
  }
  h->allocs.push_back(*p);
  return TPF_OK;
}

int validate_options(const tpf_ppe_options* o) {
  TPF_CHECK_ARG(o->method == TPF_PPE_CG || o->method == TPF_PPE_GMRES,
                "PPESolverFVMMatrixFree supports ppe_iteration_method='gmres' or 'cg' today");
  TPF_CHECK_ARG(o->precond >= TPF_PRECOND_NONE && o->precond <= TPF_PRECOND_LINE_PCR,
                "ppe_preconditioner must be 'jacobi', 'line_pcr', or 'none'");
  TPF_CHECK_ARG(!(o->method == TPF_PPE_CG && (o->precond == TPF_PRECOND_LINE || o->precond == TPF_PRECOND_LINE_PCR)),
                "ppe_iteration_method='cg' supports preconditioner='jacobi' or 'none'; line_pcr is a "
                "nonsymmetric GMRES preconditioner.");
  TPF_CHECK_ARG(o->precision == TPF_PREC_F64 || o->precision == TPF_PREC_MIXED, "unknown precision mode");
  TPF_CHECK_ARG(!(o->precision == TPF_PREC_MIXED && o->method != TPF_PPE_CG),
                "mixed precision is implemented for the CG route");
  TPF_CHECK_ARG(o->tol > 0.0 && std::isfinite(o->tol), "tolerance must be > 0");
  TPF_CHECK_ARG(o->maxiter >= 0, "maxiter must be >= 0");
  TPF_CHECK_ARG(o->restart >= 1 && o->restart <= 1024, "restart must be in [1, 1024]");
  TPF_CHECK_ARG(o->c_tau > 0.0, "c_tau must be > 0");
  TPF_CHECK_ARG(o->precond != TPF_PRECOND_LINE_PCR || o->pcr_stages >= 1, "ppe_pcr_stages must be >= 1");
  return TPF_OK;
}

LineArgs line_args(const Grid3& g, int axis) {
  LineArgs L{};
  if (axis == 0) {
    L.lines = g.n1 * g.n2; L.n = g.n0; L.stride = g.st0; L.lmod = 1 << 30; L.lstride_hi = 0; L.lstride_lo = 1;
  } else if (axis == 1) {
    L.lines = g.n0 * g.n2; L.n = g.n1; L.stride = g.n2; L.lmod = g.n2; L.lstride_hi = g.st0; L.lstride_lo = 1;
  } else {
    L.lines = g.n0 * g.n1; L.n = g.n2; L.stride = 1; L.lmod = 1 << 30; L.lstride_hi = 0; L.lstride_lo = g.n2;
  }
  return L;
}

int ensure_gmres(tpf_ppe* h) {
  int m = h->o.restart;
  if (h->V && h->V_cols >= m + 1) return TPF_OK;
  if (h->V) {
    cudaFree(h->V);
    cudaFree(h->gm);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->V), h->allocs.end());
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->gm), h->allocs.end());
  }
  int st;
  if ((st = dalloc(h, &h->V, (size_t)(m + 1) * h->g.ndof))) return st;
  size_t gm_len = (size_t)m * (m + 2) + 2 * m + (m + 1) * 4 + 8;
  if ((st = dalloc(h, &h->gm, gm_len))) return st;
  h->V_cols = m + 1;
  return TPF_OK;
}

int ew_grid(const tpf_ppe* h) { return h->ew_blocks; }

// the truncated-PCR kernels may use up to 227 KB of dynamic shared memory (set
// once, before any stream capture)
int pcr_attributes() {
  static int done_attr = 0;
  if (!done_attr) {
    TPF_CUDA_TRY(cudaFuncSetAttribute(pcr_solve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      227 * 1024));
    TPF_CUDA_TRY(cudaFuncSetAttribute(pcr_solve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      227 * 1024));
    done_attr = 1;
  }
  return TPF_OK;
}

// z = M^-1 r on the unweighted system (reference preconditioners), done-guarded
int precond_L(tpf_ppe* h, const double* r, double* z, cudaStream_t s, const int* done) {
  const Grid3& g = h->g;
  switch (h->o.precond) {
    case TPF_PRECOND_NONE:
      TPF_CUDA_TRY(cudaMemcpyAsync(z, r, sizeof(double) * g.ndof, cudaMemcpyDeviceToDevice, s));
      break;
    case TPF_PRECOND_JACOBI:
      jacobi_L_kernel<<<ew_grid(h), 256, 0, s>>>(g.ndof, g.pin, h->dinvL, r, z, done);
      break;
    case TPF_PRECOND_LINE_PCR: {
      // additive shifted line solves by truncated PCR (the reference's GPU variant)
      for (int ax = 0; ax < h->ndim; ++ax) {
        LineArgs L = line_args(g, ax);
        const int nstage = std::min(h->o.pcr_stages, (int)std::ceil(std::log2((double)std::max(L.n, 2))));
        const size_t smem = sizeof(double) * 8 * (size_t)L.n;
        TPF_CHECK_ARG(smem <= 227 * 1024, "truncated-PCR line solve: lines of %d nodes exceed shared memory", L.n);
        const double sc = (ax == h->ndim - 1) ? 1.0 / h->ndim : 1.0;
        const int ast = pcr_attributes();
        if (ast) return ast;
        if (ax == 0)
          pcr_solve_kernel<false><<<L.lines, 256, smem, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax], r, z, g.pin,
                                                              nstage, 1.0, done);
        else
          pcr_solve_kernel<true><<<L.lines, 256, smem, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax], r, z, g.pin,
                                                             nstage, sc, done);
      }
      break;
    }
    default: {
      // additive shifted line solves: z = (sum_a T_a^-1 r) / ndim, r[pin] = 0, z[pin] = 0
      for (int ax = 0; ax < h->ndim; ++ax) {
        LineArgs L = line_args(g, ax);
        const double sc = ax == h->ndim - 1 ? 1.0 / h->ndim : 1.0;
        const int wblocks = (L.lines + 3) / 4;   // one warp per line, 4 lines per block
#define TPF_THOMAS_WARP(KK)                                                                                    \
  if (ax == 0)                                                                                                 \
    thomas_warp_kernel<false, KK><<<wblocks, 128, 0, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax], r, z, g.pin, \
                                                          1.0, done);                                          \
  else                                                                                                         \
    thomas_warp_kernel<true, KK><<<wblocks, 128, 0, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax], r, z, g.pin,  \
                                                         sc, done);
        if (L.n <= 32 * 4) { TPF_THOMAS_WARP(4) }
        else if (L.n <= 32 * 9) { TPF_THOMAS_WARP(9) }
        else if (L.n <= 32 * 17) { TPF_THOMAS_WARP(17) }
        else if (L.n <= 32 * 33) { TPF_THOMAS_WARP(33) }
        else {
          const int blocks = (L.lines + 127) / 128;
          if (ax == 0)
            thomas_solve_kernel<false><<<blocks, 128, 0, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax], r, z, h->t2,
                                                              g.pin, 1.0, done);
          else
            thomas_solve_kernel<true><<<blocks, 128, 0, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax], r, z, h->t2,
                                                             g.pin, sc, done);
        }
#undef TPF_THOMAS_WARP
      }
      if (h->ndim == 1) { /* unreachable: ndim >= 2 */ }
    }
  }
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// SciPy 1.18.1 gmres restated on the device (gmres.cuh) over the FVM
// operator and the handle's preconditioner.
int solve_gmres(tpf_ppe* h, const double* rhs, double* p, const double* p_init, cudaStream_t s,
                tpf_ppe_result* res) {
  const Grid3& g = h->g;
  const int n = g.ndof;
  int st;
  cudaStreamCaptureStatus cap_state = cudaStreamCaptureStatusNone;
  TPF_CUDA_TRY(cudaStreamIsCapturing(s, &cap_state));
  TPF_CHECK_ARG(cap_state == cudaStreamCaptureStatusNone,
                "the GMRES route reads its residual on the host between restart cycles and cannot be captured "
                "into a CUDA graph (the CG route can)");
  if ((st = ensure_gmres(h))) return st;
  GmresWork W;
  W.n = n;
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
  W.w = h->z;
  W.t = h->q;
  W.exec = &h->gm_exec;
  W.cap = &h->cap;
  W.key = h->gm_key;
  // b = rhs with b[pin] = 0 ; x0 = p_init with pin = 0
  copy_pin0_kernel<<<ew_grid(h), 256, 0, s>>>(n, g.pin, rhs, W.b);
  if (p_init) copy_pin0_kernel<<<ew_grid(h), 256, 0, s>>>(n, g.pin, p_init, W.x);
  else TPF_CUDA_TRY(cudaMemsetAsync(W.x, 0, sizeof(double) * n, s));
  if (h->o.precond == TPF_PRECOND_LINE_PCR && (st = pcr_attributes())) return st;
  const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
  auto apply = [&](const double* in, double* out, cudaStream_t cs, const int* done) -> int {
    apply_L_kernel<<<ew_grid(h), 256, 0, cs>>>(g, geo, h->s[0], h->s[1], h->s[2], in, out, nullptr, done);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  };
  auto resid = [&](const double* x, double* r, cudaStream_t cs) -> int {
    apply_L_kernel<<<ew_grid(h), 256, 0, cs>>>(g, geo, h->s[0], h->s[1], h->s[2], x, r, W.b, nullptr);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  };
  auto precond = [&](const double* in, double* out, cudaStream_t cs, const int* done) -> int {
    return precond_L(h, in, out, cs, done);
  };
  GmresOutcome o;
  st = gmres_solve(W, h->o.restart, h->o.tol, h->o.maxiter, p_init != nullptr, (long long)h->o.precond,
                   (long long)h->o.pcr_stages, apply, resid, precond, s, o);
  if (st) return st;
  if (o.bnrm2 == 0.0) {
    TPF_CUDA_TRY(cudaMemsetAsync(p, 0, sizeof(double) * n, s));
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    res->refinements = 0;
    res->iterations = 0; res->applies = 0; res->rel_residual = 0.0; res->info = 0;
    return TPF_OK;
  }
  copy_pin0_kernel<<<ew_grid(h), 256, 0, s>>>(n, g.pin, W.x, p);
  TPF_CUDA_TRY(cudaGetLastError());
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  res->refinements = 0;
  res->iterations = o.inner;
  res->applies = o.applies;
  res->rel_residual = o.rnorm / o.bnrm2;
  res->info = o.converged ? 0 : (int)std::min<long long>(h->o.maxiter, 0x7fffffff);
  if (!o.converged) {
    tpf::set_error("PPESolverFVMMatrixFree did not converge cleanly (info=%d); no alternate PPE solver was applied.",
                   res->info);
    return TPF_ENOCONV;
  }
  return TPF_OK;
}

// band-resident PCG: applicable to 2-D systems whose largest node range
// (one per CTA, at least one row long) fits in the opt-in shared memory of
// one SM with 12 vectors and 6 halo rows (11 vectors and the halo in FP32
// for the mixed mode)
struct BandPlan {
  int grid, n_max;
  size_t smem;
  bool mixed;
};
bool band_plan(const tpf_ppe* h, BandPlan& bp, bool mixed) {
  if (h->cg_kernel == 1) return false;
  const Grid3& g = h->g;
  if (h->ndim != 2 || g.N2 != 0) return false;
  if (2 * g.n1 > 3 * kThreads) return false;
  const int grid = std::min(h->coop_blocks, g.ndof / g.n1);
  if (grid < 1) return false;
  const int n_max = (g.ndof + grid - 1) / grid;
  const size_t smem = mixed ? band_smem_bytes<float>(n_max, g.n1) : band_smem_bytes<double>(n_max, g.n1);
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  // static shared memory of the kernel: the reduction scratch and GridSum's flag
  if (smem + 4096 > (size_t)optin) return false;
  bp.grid = grid;
  bp.n_max = n_max;
  bp.smem = smem;
  bp.mixed = mixed;
  return true;
}

// halo buffer of a band-resident solve over `grid` blocks: [2][grid][2][3][n1]
int ensure_band_pub(tpf_ppe* h, int grid) {
  const size_t need = (size_t)2 * grid * 2 * 3 * h->g.n1;
  if (h->band_pub_len < need) {
    int st = dalloc(h, &h->band_pub, need);
    if (st) return st;
    h->band_pub_len = need;
  }
  return TPF_OK;
}

int launch_band(tpf_ppe* h, const BandPlan& bp, const Cg1Args& c, cudaStream_t s) {
  if (int st = ensure_band_pub(h, bp.grid)) return st;
  static size_t smem_set[2] = {0, 0};
  void* fn = bp.mixed ? (void*)cg1_band_kernel<float, true> : (void*)cg1_band_kernel<double, false>;
  if (bp.smem > smem_set[bp.mixed]) {
    TPF_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bp.smem));
    smem_set[bp.mixed] = bp.smem;
  }
  BandArgs a{};
  a.g = c.g;
  a.s0 = c.s64[0];
  a.s1 = c.s64[1];
  a.dinv = c.v64.dinv;
  a.s0f = c.v32.s0;
  a.s1f = c.v32.s1;
  a.dinvf = c.v32.dinv;
  a.b = c.b;
  a.x = c.x;
  a.maxiter = c.maxiter;
  a.tol = c.tol;
  a.replace_drop = c.replace_drop;
  a.x_nonzero = c.x_nonzero;
  a.n_max = bp.n_max;
  a.pub = h->band_pub;
  a.part = c.part;
  a.count = c.count;
  a.err = c.err;
  a.st = c.st;
  void* args[] = {&a};
  TPF_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(bp.grid), dim3(kThreads), args, bp.smem, s));
  return TPF_OK;
}

// Streaming PCG: the iteration as two kernels at full occupancy, chunks of
// kCgsChunk iterations replayed from a CUDA graph (see the kernels above).
constexpr int kCgsChunk = 32;

int solve_cg_stream(tpf_ppe* h, const double* rhs, double* p, const double* p_init, cudaStream_t s,
                    tpf_ppe_result* res) {
  const Grid3& g = h->g;
  const int n = g.ndof;
  int st;
  if (!h->cgs) {
    CgScal* c = nullptr;
    if ((st = dalloc(h, &c, 1))) return st;
    h->cgs = c;
  }
  CgScal* sc = static_cast<CgScal*>(h->cgs);
  cudaStreamCaptureStatus cap_state = cudaStreamCaptureStatusNone;
  TPF_CUDA_TRY(cudaStreamIsCapturing(s, &cap_state));
  const bool capturing = cap_state == cudaStreamCaptureStatusActive;
  const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
  cg_rhs_kernel<<<ew_grid(h), 256, 0, s>>>(g, geo, rhs, h->b, p_init, h->x);
  cgs_init_kernel<<<1, 1, 0, s>>>(sc, h->o.tol, h->o.maxiter, p_init ? 1 : 0);
  const bool none = (h->o.precond == TPF_PRECOND_NONE);
  const double* dinv = none ? h->ones64 : h->dinvS;
  double* r = h->c64[0];
  double* u = h->c64[1];
  double* w = h->c64[2];
  double* sv = h->c64[4];
  double* pv = h->c64[6];
  const double* s2 = (g.N2 > 0) ? h->s[2] : h->s[1];
  // stencil grid: 256 columns of the (axis 1, axis 2) plane per block, the
  // planes cut into chunks so that ~2048 threads per SM march
  const int nplane = g.st0;
  const int gx = (nplane + 255) / 256;
  const int target = 2048 * tpf::sm_count();
  int gy = std::max(1, std::min(g.n0, target / (gx * 256)));
  while (gy > 1 && gx * gy * 6 > h->part_len) --gy;
  const int chunk = (g.n0 + gy - 1) / gy;
  gy = (g.n0 + chunk - 1) / chunk;
  const int nb = gx * gy;
  TPF_CHECK_ARG(6 * nb <= h->part_len, "streaming PCG: partial-sum area too small");
  const int nr = std::max(1, std::min(h->ew_blocks, h->part_len / 8));
  const dim3 sgrid(gx, gy);
  cgs_resid_kernel<<<nr, 256, 0, s>>>(g, h->s[0], h->s[1], s2, h->b, h->x, r, h->part, sc);
  cgs_update_kernel<true><<<nb, 256, 0, s>>>(n, g.pin, dinv, w, sv, pv, h->x, r, u, h->part, sc);
  cgs_stencil_kernel<true><<<sgrid, 256, 0, s>>>(g, chunk, h->s[0], h->s[1], s2, u, pv, w, h->part, sc);
  TPF_CUDA_TRY(cudaGetLastError());
  if (capturing) {
    // inside the caller's stream capture: the iterations become a conditional
    // WHILE node of the captured graph whose body runs kCgsChunk iterations
    // and then sets the condition from the device-side state; the result is
    // read after a replay with tpf_ppe_read_result
    cudaStreamCaptureStatus cs2 = cudaStreamCaptureStatusNone;
    unsigned long long cid = 0;
    cudaGraph_t cgraph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    TPF_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs2, &cid, &cgraph, &deps, &ndeps));
    cudaGraphConditionalHandle handle;
    TPF_CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, cgraph, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t wnode;
    TPF_CUDA_TRY(cudaGraphAddNode(&wnode, cgraph, deps, ndeps, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    TPF_CUDA_TRY(cudaStreamBeginCaptureToGraph(h->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    for (int k = 0; k < kCgsChunk; ++k) {
      cgs_update_kernel<false><<<nb, 256, 0, h->cap>>>(n, g.pin, dinv, w, sv, pv, h->x, r, u, h->part, sc);
      cgs_stencil_kernel<false><<<sgrid, 256, 0, h->cap>>>(g, chunk, h->s[0], h->s[1], s2, u, pv, w, h->part, sc);
    }
    cgs_cond_kernel<<<1, 1, 0, h->cap>>>(sc, handle);
    cudaGraph_t body_out = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(h->cap, &body_out);
    if (ce != cudaSuccess) {
      cudaGetLastError();
      tpf::set_error("capturing the PCG loop body failed: %s", cudaGetErrorString(ce));
      return TPF_ECUDA;
    }
    TPF_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &wnode, 1, cudaStreamSetCaptureDependencies));
    cgs_finish_kernel<<<ew_grid(h), 256, 0, s>>>(n, g.pin, sc, h->x, p);
    TPF_CUDA_TRY(cudaGetLastError());
    h->pending = 2;
    res->iterations = -1;
    res->applies = -1;
    res->refinements = 0;
    res->rel_residual = -1.0;
    res->info = 0;
    return TPF_OK;
  }
  h->pending = 0;
  const long long key[6] = {(long long)nb * 4096 + chunk, (long long)(intptr_t)dinv, (long long)(intptr_t)h->x,
                            (long long)(intptr_t)r, (long long)n, (long long)(intptr_t)sc};
  if (!h->cg_exec || std::memcmp(h->cg_key, key, sizeof(key)) != 0) {
    if (h->cg_exec) { cudaGraphExecDestroy(h->cg_exec); h->cg_exec = nullptr; }
    if (!h->cap && cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      h->cap = nullptr;
      tpf::set_error("cudaStreamCreate failed");
      return TPF_ECUDA;
    }
    TPF_CUDA_TRY(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kCgsChunk; ++k) {
      cgs_update_kernel<false><<<nb, 256, 0, h->cap>>>(n, g.pin, dinv, w, sv, pv, h->x, r, u, h->part, sc);
      cgs_stencil_kernel<false><<<sgrid, 256, 0, h->cap>>>(g, chunk, h->s[0], h->s[1], s2, u, pv, w, h->part, sc);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(h->cap, &graph);
    if (ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      tpf::set_error("capturing the PCG iteration chunk failed: %s", cudaGetErrorString(ce));
      return TPF_ECUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&h->cg_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      h->cg_exec = nullptr;
      cudaGetLastError();
      tpf::set_error("instantiating the PCG iteration graph failed: %s", cudaGetErrorString(ie));
      return TPF_ECUDA;
    }
    std::memcpy(h->cg_key, key, sizeof(key));
  }
  CgScal hs{};
  TPF_CUDA_TRY(cudaMemcpyAsync(&hs, sc, sizeof(CgScal), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  while (!hs.done) {
    TPF_CUDA_TRY(cudaGraphLaunch(h->cg_exec, s));
    TPF_CUDA_TRY(cudaMemcpyAsync(&hs, sc, sizeof(CgScal), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
  }
  cgs_finish_kernel<<<ew_grid(h), 256, 0, s>>>(n, g.pin, sc, h->x, p);
  TPF_CUDA_TRY(cudaGetLastError());
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  res->iterations = hs.it;
  res->applies = hs.applies;
  res->refinements = 0;
  res->rel_residual = hs.bb > 0.0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
  res->info = hs.conv ? 0 : (int)std::min<long long>(h->o.maxiter, 0x7fffffff);
  if (!hs.conv) {
    tpf::set_error("PPESolverFVMMatrixFree did not converge cleanly (info=%d); no alternate PPE solver was applied.",
                   res->info);
    return TPF_ENOCONV;
  }
  return TPF_OK;
}

int solve_cg(tpf_ppe* h, const double* rhs, double* p, const double* p_init, cudaStream_t s,
             tpf_ppe_result* res) {
  const Grid3& g = h->g;
  const int n = g.ndof;
  const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
  cg_rhs_kernel<<<ew_grid(h), 256, 0, s>>>(g, geo, rhs, h->b, p_init, h->x);
  TPF_CUDA_TRY(cudaMemsetAsync(h->bar, 0, 2 * sizeof(unsigned int), s));
  TPF_CUDA_TRY(cudaMemsetAsync(h->err, 0, sizeof(int), s));
  TPF_CUDA_TRY(cudaMemsetAsync(h->st, 0, sizeof(SolveStatus), s));
  const bool none = (h->o.precond == TPF_PRECOND_NONE);
  Cg1Args a{};
  a.g = g;
  a.v64.s0 = h->s[0]; a.v64.s1 = h->s[1]; a.v64.s2 = h->s[2];
  a.v64.dinv = none ? h->ones64 : h->dinvS;
  a.v32.s0 = h->s32[0]; a.v32.s1 = h->s32[1]; a.v32.s2 = h->s32[2];
  a.v32.dinv = none ? h->ones32 : h->dinvS32;
  for (int k = 0; k < 2; ++k) {
    a.v64.r[k] = h->c64[k]; a.v64.w[k] = h->c64[2 + k]; a.v64.s[k] = h->c64[4 + k];
    a.v32.r[k] = h->c32[k]; a.v32.w[k] = h->c32[2 + k]; a.v32.s[k] = h->c32[4 + k];
  }
  a.v64.p = h->c64[6];
  a.v32.p = h->c32[6];
  a.s64[0] = h->s[0]; a.s64[1] = h->s[1]; a.s64[2] = h->s[2];
  a.b = h->b;
  a.x = h->x;
  a.tol = h->o.tol;
  a.x_nonzero = p_init ? 1 : 0;
  a.part = h->part;
  a.count = h->bar;
  a.err = h->err;
  a.st = h->st;
  const bool mixed = (h->o.precision == TPF_PREC_MIXED);
  BandPlan bp;
  const bool band = band_plan(h, bp, mixed);
  if (!mixed && (h->cg_kernel == 3 || (h->cg_kernel == 0 && !band)))
    return solve_cg_stream(h, rhs, p, p_init, s, res);
  a.maxiter = h->o.maxiter;
  a.replace_drop = h->o.inner_tol > 0.0 ? h->o.inner_tol : 1e-3;
  if (band) {
    int st = launch_band(h, bp, a, s);
    if (st) return st;
  } else {
    if (h->cg_kernel == 2) {
      tpf::set_error("the band-resident PCG needs a 2-D system whose per-SM band fits in shared memory");
      return TPF_EINVAL;
    }
    void* args[] = {&a};
    void* fn = mixed ? (void*)cg1_kernel<float, true> : (void*)cg1_kernel<double, false>;
    TPF_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(h->coop_blocks), dim3(kThreads), args, 0, s));
  }
  copy_pin0_kernel<<<ew_grid(h), 256, 0, s>>>(n, g.pin, h->x, p);
  cudaStreamCaptureStatus cap_state = cudaStreamCaptureStatusNone;
  TPF_CUDA_TRY(cudaStreamIsCapturing(s, &cap_state));
  if (cap_state == cudaStreamCaptureStatusActive) {
    // captured into the caller's graph: the status is read after a replay
    TPF_CUDA_TRY(cudaGetLastError());
    h->pending = 1;
    res->iterations = -1;
    res->applies = -1;
    res->refinements = 0;
    res->rel_residual = -1.0;
    res->info = 0;
    return TPF_OK;
  }
  h->pending = 0;
  SolveStatus hs{};
  int herr = 0;
  TPF_CUDA_TRY(cudaMemcpyAsync(&hs, h->st, sizeof(SolveStatus), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaMemcpyAsync(&herr, h->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) {
    tpf::set_error("PCG grid barrier timed out; the solve was aborted");
    return TPF_EABORT;
  }
  res->iterations = hs.iters;
  res->applies = hs.applies;
  res->refinements = hs.refinements;
  res->rel_residual = hs.bb > 0.0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
  res->info = hs.converged ? 0 : (int)std::min<long long>(h->o.maxiter, 0x7fffffff);
  if (!hs.converged) {
    tpf::set_error("PPESolverFVMMatrixFree did not converge cleanly (info=%d); no alternate PPE solver was applied.",
                   res->info);
    return TPF_ENOCONV;
  }
  return TPF_OK;
}

}  // namespace

extern "C" {

void tpf_ppe_default_options(tpf_ppe_options* o) {
  if (!o) return;
  o->method = TPF_PPE_GMRES;
  o->precond = TPF_PRECOND_LINE;
  o->precision = TPF_PREC_F64;
  o->tol = 1e-8;
  o->maxiter = 500;
  o->restart = 80;
  o->c_tau = 2.0;
  o->pcr_stages = 4;
  o->inner_tol = 1e-3;
  o->max_refine = 50;
}

int tpf_ppe_create(tpf_ppe** out, int ndim, const int64_t* N, const double* const* coords, int64_t pin,
                   const tpf_ppe_options* opts) {
  TPF_CHECK_ARG(out && N && coords, "NULL argument");
  *out = nullptr;
  TPF_CHECK_ARG(ndim == 2 || ndim == 3, "ndim must be 2 or 3");
  tpf_ppe_options o;
  tpf_ppe_default_options(&o);
  if (opts) o = *opts;
  int st = validate_options(&o);
  if (st) return st;
  int64_t nn[3] = {1, 1, 1}, ndof = 1;
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(N[a] >= 1, "N must be >= 1");
    nn[a] = N[a] + 1;
    ndof *= nn[a];
  }
  TPF_CHECK_ARG(ndof < (int64_t)1 << 31, "grid too large for 32-bit indexing");
  TPF_CHECK_ARG(pin >= 0 && pin < ndof, "pin DOF out of range");
  auto* h = new tpf_ppe();
  h->ndim = ndim;
  h->o = o;
  Grid3& g = h->g;
  g.n0 = (int)nn[0]; g.n1 = (int)nn[1]; g.n2 = (int)nn[2];
  g.N0 = (int)N[0]; g.N1 = (int)N[1]; g.N2 = ndim == 3 ? (int)N[2] : 0;
  g.st0 = g.n1 * g.n2;
  g.ndof = (int)ndof;
  g.pin = (int)pin;
  // grid metrics (fvm_matrixfree_helpers.py:23-43)
  h->h_min = INFINITY;
  std::vector<std::vector<double>> dvh(3), dfh(3);
  for (int a = 0; a < ndim; ++a) {
    std::vector<double> c(coords[a], coords[a] + nn[a]);
    std::vector<double> d(nn[a] - 1);
    for (int64_t i = 0; i + 1 < nn[a]; ++i) {
      d[i] = c[i + 1] - c[i];
      h->h_min = std::min(h->h_min, d[i]);
    }
    std::vector<double> dv(nn[a]);
    dv[0] = d[0] / 2.0;
    dv[nn[a] - 1] = d[nn[a] - 2] / 2.0;
    for (int64_t i = 1; i + 1 < nn[a]; ++i) dv[i] = (c[i + 1] - c[i - 1]) / 2.0;
    dvh[a] = dv;
    dfh[a] = d;
    h->coords.push_back(c);
  }
  auto fail = [&](int code) { tpf_ppe_destroy(h); return code; };
  for (int a = 0; a < ndim; ++a) {
    if ((st = dalloc(h, &h->dv[a], nn[a]))) return fail(st);
    if ((st = dalloc(h, &h->dface[a], nn[a] - 1))) return fail(st);
    if (cudaMemcpy(h->dv[a], dvh[a].data(), nn[a] * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->dface[a], dfh[a].data(), (nn[a] - 1) * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      tpf::set_error("copy of grid metrics failed");
      return fail(TPF_ECUDA);
    }
  }
  const size_t n = (size_t)ndof;
  for (int a = 0; a < ndim; ++a) {
    if ((st = dalloc(h, &h->s[a], n))) return fail(st);
    if ((st = dalloc(h, &h->s32[a], n))) return fail(st);
    if ((st = dalloc(h, &h->tlo[a], n))) return fail(st);
    if ((st = dalloc(h, &h->tden[a], n))) return fail(st);
    if ((st = dalloc(h, &h->tcp[a], n))) return fail(st);
  }
  if (ndim == 2) { h->s[2] = h->s[1]; h->s32[2] = h->s32[1]; }  // never read (N2 = 0)
  double** d64[] = {&h->dinvS, &h->dinvL, &h->x, &h->r, &h->z, &h->p0, &h->p1, &h->q, &h->b, &h->t1, &h->t2,
                      &h->ones64};
  for (double** pp : d64)
    if ((st = dalloc(h, pp, n))) return fail(st);
  float** d32[] = {&h->dinvS32, &h->ones32};
  for (float** pp : d32)
    if ((st = dalloc(h, pp, n))) return fail(st);
  for (int k = 0; k < 7; ++k) {
    if ((st = dalloc(h, &h->c64[k], n))) return fail(st);
    if ((st = dalloc(h, &h->c32[k], n))) return fail(st);
  }
  // ones: the identity preconditioner of the CG route ('none')
  {
    std::vector<double> ones(n, 1.0);
    std::vector<float> onesf(n, 1.0f);
    if (cudaMemcpy(h->ones64, ones.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->ones32, onesf.data(), n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      tpf::set_error("workspace init failed");
      return fail(TPF_ECUDA);
    }
  }
  // cooperative grid for the persistent PCG kernels
  int dev = 0, nsm = tpf::sm_count(), occ64 = 0, occmx = 0;
  cudaGetDevice(&dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, cg1_kernel<double, false>, kThreads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occmx, cg1_kernel<float, true>, kThreads, 0) != cudaSuccess) {
    tpf::set_error("occupancy query failed");
    return fail(TPF_ECUDA);
  }
  int per_sm = std::max(1, std::min(std::min(occ64, occmx), 1));
  int need = (int)((n + kThreads - 1) / kThreads);
  h->coop_blocks = std::max(1, std::min(nsm * per_sm, need));
  h->ew_blocks = std::max(1, std::min(nsm * 8, (int)((n + 255) / 256)));
  h->part_len = std::max(16 * h->coop_blocks, (o.restart + 2) * h->ew_blocks);
  if ((st = dalloc(h, &h->part, (size_t)h->part_len))) return fail(st);
  if ((st = dalloc(h, &h->bar, 4))) return fail(st);
  if ((st = dalloc(h, &h->err, 1))) return fail(st);
  if ((st = dalloc(h, &h->st, 1))) return fail(st);
  if ((st = dalloc(h, &h->gst, 1))) return fail(st);
  {
    // the streaming-PCG scalars and the private capture stream exist before
    // any solve, so a first solve inside a stream capture allocates nothing
    CgScal* c = nullptr;
    if ((st = dalloc(h, &c, 1))) return fail(st);
    h->cgs = c;
    if (cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      h->cap = nullptr;
      tpf::set_error("cudaStreamCreate failed");
      return fail(TPF_ECUDA);
    }
  }
  *out = h;
  return TPF_OK;
}

int tpf_ppe_destroy(tpf_ppe* h) {
  if (!h) return TPF_OK;
  if (h->gm_exec) cudaGraphExecDestroy(h->gm_exec);
  if (h->cg_exec) cudaGraphExecDestroy(h->cg_exec);
  if (h->cap) cudaStreamDestroy(h->cap);
  for (void* p : h->allocs) cudaFree(p);
  delete h;
  return TPF_OK;
}

int tpf_ppe_set_cg_kernel(tpf_ppe* h, int kind) {
  TPF_CHECK_ARG(h != nullptr, "null handle");
  TPF_CHECK_ARG(kind >= 0 && kind <= 3,
                "CG kernel must be 0 (auto), 1 (global memory), 2 (band-resident) or 3 (streaming), got %d", kind);
  h->cg_kernel = kind;
  return TPF_OK;
}

int tpf_ppe_set_options(tpf_ppe* h, const tpf_ppe_options* o) {
  TPF_CHECK_ARG(h && o, "NULL argument");
  int st = validate_options(o);
  if (st) return st;
  // the line preconditioner's state depends on c_tau and is only built when it is selected
  const bool to_line = (o->precond == TPF_PRECOND_LINE || o->precond == TPF_PRECOND_LINE_PCR);
  bool line_changed = to_line && (h->line_ready != o->precond || o->c_tau != h->o.c_tau);
  bool grow = o->restart > h->o.restart;
  h->o = *o;
  if (grow) {
    cudaFree(h->part);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->part), h->allocs.end());
    h->part_len = std::max(16 * h->coop_blocks, (o->restart + 2) * h->ew_blocks);
    if ((st = dalloc(h, &h->part, (size_t)h->part_len))) return st;
  }
  if (line_changed) h->prepared = false;
  return TPF_OK;
}

int tpf_ppe_prepare(tpf_ppe* h, const double* rho, void* stream) {
  TPF_CHECK_ARG(h && rho, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PrepArgs a{};
  a.g = h->g;
  a.geo = Geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
  a.rho = rho;
  for (int ax = 0; ax < 3; ++ax) {
    a.s[ax] = (ax < h->ndim) ? h->s[ax] : nullptr;
    a.s32[ax] = (ax < h->ndim) ? h->s32[ax] : nullptr;
    a.tlo[ax] = (ax < h->ndim) ? h->tlo[ax] : nullptr;
    a.tdg[ax] = (ax < h->ndim) ? h->tden[ax] : nullptr;
    a.tup[ax] = (ax < h->ndim) ? h->tcp[ax] : nullptr;
  }
  a.dinvS = h->dinvS;
  a.dinvS32 = h->dinvS32;
  a.dinvL = h->dinvL;
  a.shift_scale = 2.0 / (h->o.c_tau * h->h_min * h->h_min);
  a.ndim = h->ndim;
  // the shifted line systems and their Thomas factors only for the line preconditioner
  const bool line = (h->o.precond == TPF_PRECOND_LINE || h->o.precond == TPF_PRECOND_LINE_PCR);
  a.want_line = line ? 1 : 0;
  prep_faces_kernel<<<h->ew_blocks, 256, 0, s>>>(a);
  TPF_CUDA_TRY(cudaGetLastError());
  // Thomas factors for the exact line solve; truncated PCR works on the raw coefficients
  if (h->o.precond == TPF_PRECOND_LINE) {
    for (int ax = 0; ax < h->ndim; ++ax) {
      LineArgs L = line_args(h->g, ax);
      thomas_factor_kernel<<<(L.lines + 127) / 128, 128, 0, s>>>(L, h->tlo[ax], h->tden[ax], h->tcp[ax]);
    }
    TPF_CUDA_TRY(cudaGetLastError());
  }
  h->line_ready = line ? h->o.precond : 0;
  h->prepared = true;
  return TPF_OK;
}

int tpf_ppe_apply(tpf_ppe* h, const double* p, double* out, void* stream) {
  TPF_CHECK_ARG(h && p && out, "NULL argument");
  TPF_CHECK_ARG(h->prepared, "operator coefficients are not initialised (call prepare first)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
  apply_L_kernel<<<h->ew_blocks, 256, 0, s>>>(h->g, geo, h->s[0], h->s[1], h->s[2], p, out, nullptr, nullptr);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int tpf_ppe_precondition(tpf_ppe* h, const double* r, double* z, void* stream) {
  TPF_CHECK_ARG(h && r && z, "NULL argument");
  TPF_CHECK_ARG(h->prepared, "preconditioner state is not initialised (call prepare first)");
  return precond_L(h, r, z, static_cast<cudaStream_t>(stream), nullptr);
}

int tpf_ppe_solve(tpf_ppe* h, const double* rhs, const double* rho, double* p, const double* p_init, void* stream,
                  tpf_ppe_result* result) {
  TPF_CHECK_ARG(h && rhs && p, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st;
  if (rho) {
    if ((st = tpf_ppe_prepare(h, rho, stream))) return st;
  }
  TPF_CHECK_ARG(h->prepared, "operator coefficients are not initialised (call prepare first)");
  tpf_ppe_result local{};
  tpf_ppe_result* res = result ? result : &local;
  *res = tpf_ppe_result{};
  if (h->o.method == TPF_PPE_CG) return solve_cg(h, rhs, p, p_init, s, res);
  return solve_gmres(h, rhs, p, p_init, s, res);
}

int tpf_ppe_read_result(tpf_ppe* h, void* stream, tpf_ppe_result* result) {
  TPF_CHECK_ARG(h && result, "NULL argument");
  TPF_CHECK_ARG(h->pending == 1 || h->pending == 2, "no captured CG solve on this handle");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  *result = tpf_ppe_result{};
  bool conv = false;
  if (h->pending == 1) {
    SolveStatus hs{};
    int herr = 0;
    TPF_CUDA_TRY(cudaMemcpyAsync(&hs, h->st, sizeof(SolveStatus), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaMemcpyAsync(&herr, h->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) {
      tpf::set_error("PCG grid barrier timed out; the solve was aborted");
      return TPF_EABORT;
    }
    result->iterations = hs.iters;
    result->applies = hs.applies;
    result->refinements = hs.refinements;
    result->rel_residual = hs.bb > 0.0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
    conv = hs.converged != 0;
  } else {
    CgScal hs{};
    TPF_CUDA_TRY(cudaMemcpyAsync(&hs, h->cgs, sizeof(CgScal), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    result->iterations = hs.it;
    result->applies = hs.applies;
    result->rel_residual = hs.bb > 0.0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
    conv = hs.conv != 0;
  }
  result->info = conv ? 0 : (int)std::min<long long>(h->o.maxiter, 0x7fffffff);
  if (!conv) {
    tpf::set_error("PPESolverFVMMatrixFree did not converge cleanly (info=%d); no alternate PPE solver was applied.",
                   result->info);
    return TPF_ENOCONV;
  }
  return TPF_OK;
}

}  // extern "C"

namespace {

// Band-resident batch: every system 2-D and the bands of all of them resident
// at once, one block per SM.  Each system gets at least the fewest blocks
// whose largest range fits in a block's shared memory and at most one block
// per grid row (or its single-solve grid); the blocks are shared in
// proportion to the expected work, nodes x iterations ~ ndof^1.5, and trimmed
// to the SM count.
bool band_batch_plan(tpf_ppe* const* hs, int n, bool mixed, std::vector<int>& nb, std::vector<int>& nmax,
                     size_t& smem) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const size_t lim = (size_t)optin - 4096;
  auto bytes = [&](int nm, int n1) {
    return mixed ? band_smem_bytes<float>(nm, n1) : band_smem_bytes<double>(nm, n1);
  };
  const int cap = tpf::sm_count();
  std::vector<int> lo(n), hi(n);
  double wsum = 0.0;
  int sum_lo = 0;
  for (int c = 0; c < n; ++c) {
    const tpf_ppe* h = hs[c];
    const Grid3& g = h->g;
    if (h->cg_kernel == 1 || h->cg_kernel == 3 || h->ndim != 2 || g.N2 != 0 || 2 * g.n1 > 3 * kThreads)
      return false;
    hi[c] = std::min(h->coop_blocks, g.ndof / g.n1);
    int k = 1;
    while (k <= hi[c] && bytes((g.ndof + k - 1) / k, g.n1) > lim) ++k;
    if (k > hi[c]) return false;
    lo[c] = k;
    sum_lo += k;
    wsum += std::pow((double)g.ndof, 1.5);
  }
  if (sum_lo > cap) return false;
  int used = 0;
  for (int c = 0; c < n; ++c) {
    const int share = (int)((double)cap * std::pow((double)hs[c]->g.ndof, 1.5) / wsum);
    nb[c] = std::max(lo[c], std::min(hi[c], share));
    used += nb[c];
  }
  while (used > cap) {   // trim the largest shares above their minimum
    int m = -1;
    for (int c = 0; c < n; ++c)
      if (nb[c] > lo[c] && (m < 0 || nb[c] > nb[m])) m = c;
    --nb[m];
    --used;
  }
  smem = 0;
  for (int c = 0; c < n; ++c) {
    nmax[c] = (hs[c]->g.ndof + nb[c] - 1) / nb[c];
    smem = std::max(smem, bytes(nmax[c], hs[c]->g.n1));
  }
  return true;
}

// Batched streaming PCG (FP64 systems too large to keep resident): per system
// the right-hand side, the initial residual and the first iteration as the
// single-system launches, then chunks of kCgsChunk iterations of ALL systems
// in two launches each (cgsb_update_kernel / cgsb_stencil_kernel), captured
// once as a CUDA graph and replayed until no system is iterating; each
// system's blocks (threads in proportion to its nodes) return at once when
// its solve is done.  Writes p[c] and results[c]; returns the batch status.
constexpr int kBatchStencilThreads = 128;

int solve_cgs_batch(tpf_ppe* const* hs, int n, const double* const* rhs, double* const* p, cudaStream_t s,
                    tpf_ppe_result* results) {
  int st;
  std::unique_ptr<CgsBatch> b(new CgsBatch());
  b->n = n;
  b->first[0] = 0;
  long long tot = 0;
  for (int c = 0; c < n; ++c) tot += hs[c]->g.ndof;
  const long long target = 2048LL * tpf::sm_count();   // threads resident at once
  for (int c = 0; c < n; ++c) {
    tpf_ppe* h = hs[c];
    const Grid3& g = h->g;
    if (!h->cgs) {
      CgScal* cs = nullptr;
      if ((st = dalloc(h, &cs, 1))) return st;
      h->cgs = cs;
    }
    CgScal* sc = static_cast<CgScal*>(h->cgs);
    // stencil blocks of kBatchStencilThreads columns (fewer idle lanes on the
    // short rows of the smaller systems than 256-column blocks)
    const int gx = (g.st0 + kBatchStencilThreads - 1) / kBatchStencilThreads;
    const long long want =
        std::max<long long>((long long)kBatchStencilThreads * gx, target * g.ndof / std::max<long long>(tot, 1));
    int gy = (int)std::max<long long>(1, std::min<long long>(g.n0, want / ((long long)kBatchStencilThreads * gx)));
    while (gy > 1 && gx * gy * 6 > h->part_len) --gy;
    const int chunk = (g.n0 + gy - 1) / gy;
    gy = (g.n0 + chunk - 1) / chunk;
    TPF_CHECK_ARG(6 * gx * gy <= h->part_len, "batched streaming PCG: partial-sum area of system %d too small", c);
    CgsSys& y = b->c[c];
    y.g = g;
    y.chunk = chunk;
    y.gx = gx;
    y.gy = gy;
    y.s0 = h->s[0];
    y.s1 = h->s[1];
    y.s2 = (g.N2 > 0) ? h->s[2] : h->s[1];
    y.dinv = (h->o.precond == TPF_PRECOND_NONE) ? h->ones64 : h->dinvS;
    y.x = h->x;
    y.r = h->c64[0];
    y.u = h->c64[1];
    y.w = h->c64[2];
    y.sv = h->c64[4];
    y.pv = h->c64[6];
    y.part = h->part;
    y.sc = sc;
    b->first[c + 1] = b->first[c] + gx * gy;
    const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
    cg_rhs_kernel<<<ew_grid(h), 256, 0, s>>>(g, geo, rhs[c], h->b, nullptr, h->x);
    cgs_init_kernel<<<1, 1, 0, s>>>(sc, h->o.tol, h->o.maxiter, 0);
    const int nr = std::max(1, std::min(h->ew_blocks, h->part_len / 8));
    cgs_resid_kernel<<<nr, 256, 0, s>>>(g, y.s0, y.s1, y.s2, h->b, h->x, y.r, y.part, sc);
    cgs_update_kernel<true><<<gx * gy, 256, 0, s>>>(g.ndof, g.pin, y.dinv, y.w, y.sv, y.pv, y.x, y.r, y.u, y.part,
                                                     sc);
    cgs_stencil_kernel<true><<<dim3(gx, gy), kBatchStencilThreads, 0, s>>>(g, chunk, y.s0, y.s1, y.s2, y.u, y.pv,
                                                                            y.w, y.part, sc);
    TPF_CUDA_TRY(cudaGetLastError());
  }
  tpf_ppe* h0 = hs[0];
  if (!h0->batch_pending && (st = dalloc(h0, &h0->batch_pending, 1))) return st;
  if (!h0->cap && cudaStreamCreateWithFlags(&h0->cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    h0->cap = nullptr;
    tpf::set_error("cudaStreamCreate failed");
    return TPF_ECUDA;
  }
  const int nblk = b->first[n];
  TPF_CUDA_TRY(cudaStreamBeginCapture(h0->cap, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < kCgsChunk; ++k) {
    cgsb_update_kernel<<<nblk, 256, 0, h0->cap>>>(*b);
    cgsb_stencil_kernel<<<nblk, kBatchStencilThreads, 0, h0->cap>>>(*b);
  }
  cgsb_pending_kernel<<<1, 64, 0, h0->cap>>>(*b, h0->batch_pending);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h0->cap, &graph);
  if (ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    tpf::set_error("capturing the batched PCG chunk failed: %s", cudaGetErrorString(ce));
    return TPF_ECUDA;
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    cudaGetLastError();
    tpf::set_error("instantiating the batched PCG graph failed: %s", cudaGetErrorString(ie));
    return TPF_ECUDA;
  }
  cgsb_pending_kernel<<<1, 64, 0, s>>>(*b, h0->batch_pending);
  int pending = 0;
  cudaError_t le = cudaMemcpyAsync(&pending, h0->batch_pending, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (le == cudaSuccess) le = cudaStreamSynchronize(s);
  while (le == cudaSuccess && pending > 0) {
    le = cudaGraphLaunch(exec, s);
    if (le == cudaSuccess) le = cudaMemcpyAsync(&pending, h0->batch_pending, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (le == cudaSuccess) le = cudaStreamSynchronize(s);
  }
  cudaGraphExecDestroy(exec);
  TPF_CUDA_TRY(le);
  std::vector<CgScal> hsc(n);
  for (int c = 0; c < n; ++c) {
    tpf_ppe* h = hs[c];
    cgs_finish_kernel<<<ew_grid(h), 256, 0, s>>>(h->g.ndof, h->g.pin, b->c[c].sc, h->x, p[c]);
    TPF_CUDA_TRY(cudaMemcpyAsync(&hsc[c], b->c[c].sc, sizeof(CgScal), cudaMemcpyDeviceToHost, s));
  }
  TPF_CUDA_TRY(cudaGetLastError());
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  int status = TPF_OK;
  for (int c = 0; c < n; ++c) {
    tpf_ppe_result r{};
    r.iterations = hsc[c].it;
    r.applies = hsc[c].applies;
    r.refinements = 0;
    r.rel_residual = hsc[c].bb > 0.0 ? std::sqrt(hsc[c].rr / hsc[c].bb) : 0.0;
    r.info = hsc[c].conv ? 0 : (int)std::min<long long>(hs[c]->o.maxiter, 0x7fffffff);
    if (results) results[c] = r;
    if (!hsc[c].conv && status == TPF_OK) {
      tpf::set_error("batched PCG system %d did not converge (info=%d)", c, r.info);
      status = TPF_ENOCONV;
    }
  }
  return status;
}

int launch_band_batch(tpf_ppe* const* hs, int n, const double* const* rhs, bool mixed, const std::vector<int>& nb,
                      const std::vector<int>& nmax, size_t smem, cudaStream_t s) {
  auto* b = new BandBatch();
  b->n = n;
  b->first[0] = 0;
  for (int c = 0; c < n; ++c) {
    tpf_ppe* h = hs[c];
    if (int st = ensure_band_pub(h, nb[c])) { delete b; return st; }
    const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
    cg_rhs_kernel<<<ew_grid(h), 256, 0, s>>>(h->g, geo, rhs[c], h->b, nullptr, h->x);
    cudaMemsetAsync(h->bar, 0, 2 * sizeof(unsigned int), s);
    cudaMemsetAsync(h->err, 0, sizeof(int), s);
    cudaMemsetAsync(h->st, 0, sizeof(SolveStatus), s);
    const bool none = (h->o.precond == TPF_PRECOND_NONE);
    BandArgs& a = b->c[c];
    a = BandArgs{};
    a.g = h->g;
    a.s0 = h->s[0];
    a.s1 = h->s[1];
    a.dinv = none ? h->ones64 : h->dinvS;
    a.s0f = h->s32[0];
    a.s1f = h->s32[1];
    a.dinvf = none ? h->ones32 : h->dinvS32;
    a.b = h->b;
    a.x = h->x;
    a.maxiter = h->o.maxiter;
    a.tol = h->o.tol;
    a.replace_drop = h->o.inner_tol > 0.0 ? h->o.inner_tol : 1e-3;
    a.x_nonzero = 0;
    a.n_max = nmax[c];
    a.pub = h->band_pub;
    a.part = h->part;
    a.count = h->bar;
    a.err = h->err;
    a.st = h->st;
    b->first[c + 1] = b->first[c] + nb[c];
  }
  void* fn = mixed ? (void*)cg1_band_batch_kernel<float, true> : (void*)cg1_band_batch_kernel<double, false>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    void* args[] = {b};
    e = cudaLaunchCooperativeKernel(fn, dim3(b->first[n]), dim3(kThreads), args, smem, s);
  }
  delete b;
  TPF_CUDA_TRY(e);
  return TPF_OK;
}

}  // namespace

extern "C" {

int tpf_ppe_solve_batched(tpf_ppe* const* hs, int n, const double* const* rhs, const double* const* rho,
                          double* const* p, void* stream, tpf_ppe_result* results) {
  TPF_CHECK_ARG(hs && rhs && p && n >= 1, "NULL argument or empty batch");
  TPF_CHECK_ARG(n <= kBatchMax, "at most %d systems per batched solve (got %d)", kBatchMax, n);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st;
  const bool mixed = hs[0]->o.precision == TPF_PREC_MIXED;
  for (int c = 0; c < n; ++c) {
    tpf_ppe* h = hs[c];
    TPF_CHECK_ARG(h && rhs[c] && p[c], "NULL handle or array for system %d", c);
    TPF_CHECK_ARG(h->o.method == TPF_PPE_CG, "batched solves run the CG route (system %d)", c);
    TPF_CHECK_ARG((h->o.precision == TPF_PREC_MIXED) == mixed, "all systems of a batch share one precision");
    if (rho && rho[c] && (st = tpf_ppe_prepare(h, rho[c], stream))) return st;
    TPF_CHECK_ARG(h->prepared, "operator coefficients of system %d are not initialised", c);
  }
  // the band-resident batch where every band fits at once, else the
  // all-global persistent body
  std::vector<int> bnb(n), bnmax(n);
  size_t bsmem = 0;
  bool force_band = false;
  for (int c = 0; c < n; ++c) force_band = force_band || hs[c]->cg_kernel == 2;
  bool force_global = false, force_stream = false;
  for (int c = 0; c < n; ++c) {
    force_global = force_global || hs[c]->cg_kernel == 1;
    force_stream = force_stream || hs[c]->cg_kernel == 3;
  }
  TPF_CHECK_ARG(!(force_stream && (force_band || force_global)), "conflicting CG kernel choices in one batch");
  TPF_CHECK_ARG(!(force_stream && mixed), "the batched streaming PCG runs FP64 systems");
  if (force_stream) return solve_cgs_batch(hs, n, rhs, p, s, results);
  if (band_batch_plan(hs, n, mixed, bnb, bnmax, bsmem)) {
    if ((st = launch_band_batch(hs, n, rhs, mixed, bnb, bnmax, bsmem, s))) return st;
  } else if (force_band) {
    tpf::set_error("the band-resident batch needs 2-D systems whose bands all fit in shared memory at once");
    return TPF_EINVAL;
  } else if (!mixed && !force_global) {
    return solve_cgs_batch(hs, n, rhs, p, s, results);
  } else {
    double wsum = 0.0;
    for (int c = 0; c < n; ++c) wsum += std::pow((double)hs[c]->g.ndof, 1.5);
    // blocks: one per SM (the kernel's occupancy), shared in proportion to the
    // expected work, nodes x iterations ~ ndof^1.5 (Jacobi-PCG iteration counts
    // grow like the grid's linear size)
    void* fn = mixed ? (void*)cg1_batch_kernel<float, true> : (void*)cg1_batch_kernel<double, false>;
    int per_sm = 0;
    TPF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0));
    const int cap = tpf::sm_count() * std::max(1, per_sm);
    TPF_CHECK_ARG(n <= cap, "batch of %d systems exceeds the %d co-resident blocks", n, cap);
    std::vector<int> nb(n);
    int used = 0;
    for (int c = 0; c < n; ++c) {
      const double share = (double)cap * std::pow((double)hs[c]->g.ndof, 1.5) / wsum;
      nb[c] = std::max(1, std::min(hs[c]->coop_blocks, (int)share));
      used += nb[c];
    }
    while (used > cap) {   // trim the largest shares
      int m = 0;
      for (int c = 1; c < n; ++c)
        if (nb[c] > nb[m]) m = c;
      --nb[m];
      --used;
    }
    auto* b = new Cg1Batch();
    b->n = n;
    b->first[0] = 0;
    for (int c = 0; c < n; ++c) {
      tpf_ppe* h = hs[c];
      const Geo geo{{h->dv[0], h->dv[1], h->dv[2]}, {h->dface[0], h->dface[1], h->dface[2]}};
      cg_rhs_kernel<<<ew_grid(h), 256, 0, s>>>(h->g, geo, rhs[c], h->b, nullptr, h->x);
      TPF_CUDA_TRY(cudaMemsetAsync(h->bar, 0, 2 * sizeof(unsigned int), s));
      TPF_CUDA_TRY(cudaMemsetAsync(h->err, 0, sizeof(int), s));
      TPF_CUDA_TRY(cudaMemsetAsync(h->st, 0, sizeof(SolveStatus), s));
      Cg1Args& a = b->c[c];
      a = Cg1Args{};
      a.g = h->g;
      const bool none = (h->o.precond == TPF_PRECOND_NONE);
      a.v64.s0 = h->s[0]; a.v64.s1 = h->s[1]; a.v64.s2 = h->s[2];
      a.v64.dinv = none ? h->ones64 : h->dinvS;
      a.v32.s0 = h->s32[0]; a.v32.s1 = h->s32[1]; a.v32.s2 = h->s32[2];
      a.v32.dinv = none ? h->ones32 : h->dinvS32;
      for (int k = 0; k < 2; ++k) {
        a.v64.r[k] = h->c64[k]; a.v64.w[k] = h->c64[2 + k]; a.v64.s[k] = h->c64[4 + k];
        a.v32.r[k] = h->c32[k]; a.v32.w[k] = h->c32[2 + k]; a.v32.s[k] = h->c32[4 + k];
      }
      a.v64.p = h->c64[6];
      a.v32.p = h->c32[6];
      a.s64[0] = h->s[0]; a.s64[1] = h->s[1]; a.s64[2] = h->s[2];
      a.b = h->b;
      a.x = h->x;
      a.tol = h->o.tol;
      a.x_nonzero = 0;
      a.part = h->part;
      a.count = h->bar;
      a.err = h->err;
      a.st = h->st;
      a.maxiter = h->o.maxiter;
      a.replace_drop = h->o.inner_tol > 0.0 ? h->o.inner_tol : 1e-3;
      b->first[c + 1] = b->first[c] + nb[c];
    }
    void* args[] = {b};
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(b->first[n]), dim3(kThreads), args, 0, s);
    delete b;
    TPF_CUDA_TRY(e);
  }
  std::vector<SolveStatus> hst(n);
  std::vector<int> herr(n);
  for (int c = 0; c < n; ++c) {
    tpf_ppe* h = hs[c];
    copy_pin0_kernel<<<ew_grid(h), 256, 0, s>>>(h->g.ndof, h->g.pin, h->x, p[c]);
    TPF_CUDA_TRY(cudaMemcpyAsync(&hst[c], h->st, sizeof(SolveStatus), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaMemcpyAsync(&herr[c], h->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  }
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  int status = TPF_OK;
  for (int c = 0; c < n; ++c) {
    tpf_ppe_result r{};
    r.iterations = hst[c].iters;
    r.applies = hst[c].applies;
    r.refinements = hst[c].refinements;
    r.rel_residual = hst[c].bb > 0.0 ? std::sqrt(hst[c].rr / hst[c].bb) : 0.0;
    r.info = hst[c].converged ? 0 : (int)std::min<long long>(hs[c]->o.maxiter, 0x7fffffff);
    if (results) results[c] = r;
    if (herr[c]) {
      tpf::set_error("PCG barrier of batched system %d timed out; the solve was aborted", c);
      status = TPF_EABORT;
    } else if (!hst[c].converged && status == TPF_OK) {
      tpf::set_error("batched PCG system %d did not converge (info=%d)", c, r.info);
      status = TPF_ENOCONV;
    }
  }
  return status;
}

}  // extern "C"

namespace tpf {

int ppe_view(tpf_ppe* h, PpeView* v) {
  TPF_CHECK_ARG(h && v, "NULL argument");
  v->ndim = h->ndim;
  v->n0 = h->g.n0; v->n1 = h->g.n1; v->n2 = h->g.n2;
  v->N0 = h->g.N0; v->N1 = h->g.N1; v->N2 = h->g.N2;
  v->ndof = h->g.ndof;
  v->pin = h->g.pin;
  for (int a = 0; a < 3; ++a) {
    v->s[a] = h->s[a];
    v->dv[a] = h->dv[a];
  }
  v->dinvS = h->dinvS;
  v->prepared = h->prepared;
  return TPF_OK;
}

int ppe_options(tpf_ppe* h, tpf_ppe_options* o) {
  TPF_CHECK_ARG(h && o, "NULL argument");
  *o = h->o;
  return TPF_OK;
}

}  // namespace tpf

// ---- allocation-free CG solve ----------------------------------------------------
//
// For callers that must not allocate device memory while they run: a host
// whose caching allocator (PyTorch's, or a memory pool) already holds the
// device memory, so that a cudaMalloc inside a time step can fail or stall;
// solver loops with a fixed memory budget checked at start-up.  The whole
// workspace lives in one file-scope device array of fixed size; the entry
// point issues no cudaMalloc / cudaFree and calls no allocating library.
// Every call on a device uses the same array: calls that overlap in time on
// one device (two host threads, or two streams without ordering) race on it.

namespace {

constexpr int kStaticMaxDof = TPF_PPE_STATIC_MAX_DOF;
constexpr int kStaticMaxAxis = TPF_PPE_STATIC_MAX_AXIS;
constexpr int kStaticMaxBlocks = 256;
// layout in doubles: coords | dv | dface (3 x kStaticMaxAxis each), s0..s2,
// dinvS, dinvL, b, x, ones, c64[7] (kStaticMaxDof each), s32[3] + dinvS32
// (4 x kStaticMaxDof floats), partial sums, then 32 doubles for counter /
// error flag / status
constexpr size_t kStaticAxisDoubles = (size_t)9 * kStaticMaxAxis;
constexpr size_t kStaticVecDoubles = (size_t)15 * kStaticMaxDof;
constexpr size_t kStaticF32Doubles = (size_t)2 * kStaticMaxDof;
constexpr size_t kStaticPartDoubles = (size_t)16 * kStaticMaxBlocks;
constexpr size_t kStaticDoubles = kStaticAxisDoubles + kStaticVecDoubles + kStaticF32Doubles + kStaticPartDoubles + 32;
static_assert(sizeof(SolveStatus) <= 16 * sizeof(double), "status slot too small");

static __device__ __align__(256) double g_static_ws[kStaticDoubles];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_ptr[kStaticMaxDevices] = {};

// Device address of g_static_ws for the current device, looked up once per
// device (the first call on a device does the lookup; later calls reuse it).
// Under lazy module loading the lookup also loads the module, which reserves
// the array's device memory.  A cudaDeviceReset invalidates the kept address.
int static_workspace(double** out) {
  int dev = -1;
  TPF_CUDA_TRY(cudaGetDevice(&dev));
  TPF_CHECK_ARG(dev >= 0 && dev < kStaticMaxDevices, "device ordinal out of range for the static workspace");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_ws);
    if (e != cudaSuccess || p == nullptr) {
      tpf::set_error("cudaGetSymbolAddress of the static PPE workspace failed: %s", cudaGetErrorString(e));
      return TPF_ECUDA;
    }
    g_static_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_static_ptr[dev];
  return TPF_OK;
}

// node control-volume widths and face widths from node coordinates
// (fvm_matrixfree_helpers.py:23-43), same arithmetic as tpf_ppe_create
__global__ void static_metrics_kernel(const double* c, double* dv, double* dface, int nn) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    if (i + 1 < nn) dface[i] = c[i + 1] - c[i];
    double v;
    if (i == 0) v = (c[1] - c[0]) / 2.0;
    else if (i == nn - 1) v = (c[nn - 1] - c[nn - 2]) / 2.0;
    else v = (c[i + 1] - c[i - 1]) / 2.0;
    dv[i] = v;
  }
}

__global__ void static_fill_kernel(double* x, int n, double v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

}  // namespace

extern "C" int tpf_ppe_solve_cg_static(int ndim, const int64_t* N, const double* const* coords, int64_t pin,
                                       const double* rhs, const double* rho, double* p, const double* p_init,
                                       int precond, double tol, int64_t maxiter, void* stream,
                                       tpf_ppe_result* result) {
  TPF_CHECK_ARG(N && coords && rhs && rho && p, "NULL argument");
  TPF_CHECK_ARG(ndim == 2 || ndim == 3, "ndim must be 2 or 3");
  TPF_CHECK_ARG(precond == TPF_PRECOND_JACOBI || precond == TPF_PRECOND_NONE,
                "the static-workspace CG solve supports preconditioner 'jacobi' or 'none'");
  TPF_CHECK_ARG(tol > 0.0 && std::isfinite(tol), "tolerance must be > 0");
  TPF_CHECK_ARG(maxiter >= 0, "maxiter must be >= 0");
  int64_t nn[3] = {1, 1, 1}, ndof = 1;
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(N[a] >= 1, "N must be >= 1");
    TPF_CHECK_ARG(coords[a] != nullptr, "NULL coordinate array");
    nn[a] = N[a] + 1;
    if (nn[a] > kStaticMaxAxis) {
      tpf::set_error("static-workspace CG solve: %lld nodes on axis %d exceeds the maximum of %d",
                     (long long)nn[a], a, kStaticMaxAxis);
      return TPF_EINVAL;
    }
    ndof *= nn[a];
  }
  if (ndof > kStaticMaxDof) {
    tpf::set_error("static-workspace CG solve: %lld nodes exceed the maximum of %d (use tpf_ppe_create/tpf_ppe_solve)",
                   (long long)ndof, kStaticMaxDof);
    return TPF_EINVAL;
  }
  TPF_CHECK_ARG(pin >= 0 && pin < ndof, "pin DOF out of range");
  double* ws = nullptr;
  int st = static_workspace(&ws);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = (int)ndof;
  Grid3 g{};
  g.n0 = (int)nn[0]; g.n1 = (int)nn[1]; g.n2 = (int)nn[2];
  g.N0 = (int)N[0]; g.N1 = (int)N[1]; g.N2 = ndim == 3 ? (int)N[2] : 0;
  g.st0 = g.n1 * g.n2;
  g.ndof = n;
  g.pin = (int)pin;
  // carve the workspace
  double* cur = ws;
  double *cst[3], *dv[3], *dface[3];
  for (int a = 0; a < 3; ++a) { cst[a] = cur; cur += kStaticMaxAxis; }
  for (int a = 0; a < 3; ++a) { dv[a] = cur; cur += kStaticMaxAxis; }
  for (int a = 0; a < 3; ++a) { dface[a] = cur; cur += kStaticMaxAxis; }
  double* sv[3];
  for (int a = 0; a < 3; ++a) { sv[a] = cur; cur += kStaticMaxDof; }
  double* dinvS = cur; cur += kStaticMaxDof;
  double* dinvL = cur; cur += kStaticMaxDof;
  double* b = cur; cur += kStaticMaxDof;
  double* x = cur; cur += kStaticMaxDof;
  double* ones = cur; cur += kStaticMaxDof;
  double* c64[7];
  for (int k = 0; k < 7; ++k) { c64[k] = cur; cur += kStaticMaxDof; }
  float* f32 = reinterpret_cast<float*>(cur);
  float* s32[3] = {f32, f32 + kStaticMaxDof, f32 + 2 * (size_t)kStaticMaxDof};
  float* dinvS32 = f32 + 3 * (size_t)kStaticMaxDof;
  cur += kStaticF32Doubles;
  double* part = cur; cur += kStaticPartDoubles;
  unsigned int* bar = reinterpret_cast<unsigned int*>(cur);        // 4 counters (2 doubles)
  int* err = reinterpret_cast<int*>(cur + 2);                       // 1 flag (1 double)
  SolveStatus* stp = reinterpret_cast<SolveStatus*>(cur + 4);       // 16 doubles
  const int nsm = tpf::sm_count();
  const int ew_blocks = std::max(1, std::min(nsm * 8, (n + 255) / 256));
  const int coop_blocks = std::max(1, std::min(nsm, (n + kThreads - 1) / kThreads));
  TPF_CHECK_ARG(coop_blocks <= kStaticMaxBlocks, "cooperative grid larger than the static partial-sum area");
  // grid metrics from the host coordinates
  for (int a = 0; a < ndim; ++a) {
    TPF_CUDA_TRY(cudaMemcpyAsync(cst[a], coords[a], nn[a] * sizeof(double), cudaMemcpyHostToDevice, s));
    static_metrics_kernel<<<(int)((nn[a] + 255) / 256), 256, 0, s>>>(cst[a], dv[a], dface[a], (int)nn[a]);
  }
  const Geo geo{{dv[0], dv[1], dv[2]}, {dface[0], dface[1], dface[2]}};
  // face couplings and Jacobi diagonal (the FP32 copies are written too; unused here)
  PrepArgs pa{};
  pa.g = g;
  pa.geo = geo;
  pa.rho = rho;
  for (int a = 0; a < 3; ++a) {
    pa.s[a] = (a < ndim) ? sv[a] : nullptr;
    pa.s32[a] = (a < ndim) ? s32[a] : nullptr;
  }
  pa.dinvS = dinvS;
  pa.dinvS32 = dinvS32;
  pa.dinvL = dinvL;
  pa.shift_scale = 0.0;
  pa.ndim = ndim;
  pa.want_line = 0;
  prep_faces_kernel<<<ew_blocks, 256, 0, s>>>(pa);
  if (precond == TPF_PRECOND_NONE) static_fill_kernel<<<ew_blocks, 256, 0, s>>>(ones, n, 1.0);
  cg_rhs_kernel<<<ew_blocks, 256, 0, s>>>(g, geo, rhs, b, p_init, x);
  TPF_CUDA_TRY(cudaGetLastError());
  // the grid-barrier counter, the error flag and the status start at zero
  TPF_CUDA_TRY(cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned int), s));
  TPF_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
  TPF_CUDA_TRY(cudaMemsetAsync(stp, 0, sizeof(SolveStatus), s));
  Cg1Args a{};
  a.g = g;
  a.v64.s0 = sv[0]; a.v64.s1 = sv[1]; a.v64.s2 = (ndim == 3) ? sv[2] : sv[1];
  a.v64.dinv = (precond == TPF_PRECOND_NONE) ? ones : dinvS;
  for (int k = 0; k < 2; ++k) { a.v64.r[k] = c64[k]; a.v64.w[k] = c64[2 + k]; a.v64.s[k] = c64[4 + k]; }
  a.v64.p = c64[6];
  a.s64[0] = sv[0]; a.s64[1] = sv[1]; a.s64[2] = (ndim == 3) ? sv[2] : sv[1];
  a.b = b;
  a.x = x;
  a.tol = tol;
  a.maxiter = maxiter;
  a.replace_drop = 1e-3;
  a.x_nonzero = p_init ? 1 : 0;
  a.part = part;
  a.count = bar;
  a.err = err;
  a.st = stp;
  void* args[] = {&a};
  TPF_CUDA_TRY(cudaLaunchCooperativeKernel((void*)cg1_kernel<double, false>, dim3(coop_blocks), dim3(kThreads), args,
                                           0, s));
  copy_pin0_kernel<<<ew_blocks, 256, 0, s>>>(n, g.pin, x, p);
  TPF_CUDA_TRY(cudaGetLastError());
  SolveStatus hs{};
  int herr = 0;
  TPF_CUDA_TRY(cudaMemcpyAsync(&hs, stp, sizeof(SolveStatus), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) {
    tpf::set_error("PCG grid barrier timed out; the solve was aborted");
    return TPF_EABORT;
  }
  tpf_ppe_result local{};
  tpf_ppe_result* res = result ? result : &local;
  *res = tpf_ppe_result{};
  res->iterations = hs.iters;
  res->applies = hs.applies;
  res->refinements = 0;
  res->rel_residual = hs.bb > 0.0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
  res->info = hs.converged ? 0 : (int)std::min<long long>(maxiter, 0x7fffffff);
  if (!hs.converged) {
    tpf::set_error("PPESolverFVMMatrixFree did not converge cleanly (info=%d); no alternate PPE solver was applied.",
                   res->info);
    return TPF_ENOCONV;
  }
  return TPF_OK;
}

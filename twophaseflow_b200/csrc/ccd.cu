// CCD operator for sm_100a: batched 2x2 block-tridiagonal line solves.
//
// Each line (all lines perpendicular to the axis) solves the CCD system of the
// reference (src/twophase/ccd/ccd_solver.py:11-22, coefficients :70-76):
//   Eq-I : a1 (f'_{i-1}+f'_{i+1}) + f'_i - b1 h (f''_{i+1}-f''_{i-1}) = a1/h (f_{i+1}-f_{i-1})
//   Eq-II: b2 (f''_{i-1}+f''_{i+1}) + f''_i - b2/h (f'_{i+1}-f'_{i-1}) = a2/h^2 (f_{i-1}-2f_i+f_{i+1})
// Wall axes fold the one-sided closure into the first/last block rows
// (ccd_solver_helpers.py:227-245); periodic axes are block-circulant
// (ccd_solver_helpers.py:406-423).
//
// Algorithm (this file's own design, not the reference's dense LU):
// the block matrix is the same for every line, so its 2x2 block-LU factors
// (block_tridiag.py:67-104) are computed once on the host.  Every line is cut
// into P chunks of C rows; each chunk runs the forward/backward block-Thomas
// sweeps locally, and the exact coupling between chunks is restored by a short
// scan over the chunk carries (the sweeps are affine first-order recurrences
// whose chunk transfer matrices Phi/Psi are precomputed).  Away from the wall
// rows the factors equal the fixed point of the block Riccati recurrence, so
// only chunk 0 needs per-row tables.  A periodic axis uses the Wiener-Hopf
// factorization A = (I + Lf S^-1) LU (I + H S) of the circulant matrix and
// closes the two recurrences on the ring with (I - T_ring)^-1.
//
// Threads of a CTA: TL consecutive lines x P chunks (lines fastest), so for a
// strided axis the lanes of a warp read consecutive addresses; for the
// contiguous axis the TL lines are staged through shared memory first.
#include "tpf_common.cuh"

#include <cmath>
#include <vector>
#include <array>
#include <algorithm>

namespace {

constexpr double kAlpha1 = 7.0 / 16.0, kA1 = 15.0 / 16.0, kB1 = 1.0 / 16.0;
constexpr double kBeta2 = -1.0 / 8.0, kA2 = 3.0, kB2 = -9.0 / 8.0;

using M2 = std::array<double, 4>;  // row-major 2x2
inline M2 mul(const M2& a, const M2& b) {
  return {a[0] * b[0] + a[1] * b[2], a[0] * b[1] + a[1] * b[3],
          a[2] * b[0] + a[3] * b[2], a[2] * b[1] + a[3] * b[3]};
}
inline M2 sub(const M2& a, const M2& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2], a[3] - b[3]}; }
inline M2 add(const M2& a, const M2& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2], a[3] + b[3]}; }
inline M2 neg(const M2& a) { return {-a[0], -a[1], -a[2], -a[3]}; }
inline double det(const M2& a) { return a[0] * a[3] - a[1] * a[2]; }
inline M2 inv(const M2& a) {
  double d = det(a), id = 1.0 / d;
  return {a[3] * id, -a[1] * id, -a[2] * id, a[0] * id};
}
inline M2 eye() { return {1.0, 0.0, 0.0, 1.0}; }
inline double maxabs(const M2& a) {
  return std::max(std::max(std::fabs(a[0]), std::fabs(a[1])), std::max(std::fabs(a[2]), std::fabs(a[3])));
}

// Table layout (doubles), C = chunk length.
struct TabLayout {
  int C;
  __host__ __device__ int lf0() const { return 0; }
  __host__ __device__ int p0() const { return 4 * C; }
  __host__ __device__ int h0() const { return 8 * C; }
  __host__ __device__ int psi0() const { return 12 * C; }
  __host__ __device__ int phi() const { return 16 * C; }
  __host__ __device__ int psi() const { return 20 * C; }          // C+1 entries
  __host__ __device__ int cst() const { return 24 * C + 4; }      // Lfi, Pi, Hi, Plast, Gf, Gb
  __host__ __device__ int bc() const { return cst() + 24; }       // L0 UN Ml Mr cIl cIr cII(6) c1 c2
  __host__ __device__ int total() const { return bc() + 32; }
};

}  // namespace

struct tpf_ccd_plan {
  int64_t n_pts = 0;
  double h = 0.0;
  int bc = TPF_BC_WALL;
  int dtype = TPF_F64;
  int n_rows = 0, C = 32, P = 1;
  double* d_tab = nullptr;   // double table
  float* d_tabf = nullptr;   // float copy (interior factors for F32)
  double* d_J = nullptr;     // metric J, dJ (n_pts each)
  bool has_metric = false;
};

namespace {

struct CcdArgs {
  const void* f;
  void* d1;
  void* d2;
  int64_t outer, inner, n_lines;
  int n, n_rows, C, P, TL;
  int LS, FS;             // ybuf / staged-f line strides (elements)
  int tab_total;
  const double* tab;      // double table (closures)
  const void* tabT;       // table in compute type
  const double* J;        // metric or nullptr
  int ovl, ovr;           // wall closure overrides (left / right)
  double bcl0, bcl1, bcr0, bcr1;
};

template <typename T>
struct V2 { T a, b; };

template <typename T>
__device__ __forceinline__ V2<T> mv(const T* m, V2<T> v) {
  return {m[0] * v.a + m[1] * v.b, m[2] * v.a + m[3] * v.b};
}

// f value at node k of line with base offset `base` and stride `st`.
template <typename T, bool STAGED>
__device__ __forceinline__ T load_f(const T* __restrict__ f, const T* fs, int64_t base, int64_t st,
                                    int k, bool valid) {
  if (STAGED) return fs[k];
  return valid ? __ldg(f + base + (int64_t)k * st) : T(0);
}

template <typename T, bool PERIODIC, bool STAGED>
__global__ void __launch_bounds__(512) ccd_line_kernel(CcdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TL = a.TL, C = a.C, P = a.P, n = a.n, n_rows = a.n_rows;
  const TabLayout lay{C};
  // shared layout: tab(T) | ybuf(T) | fs(T, staged) | cin(T) | cinb(T) | bcs(double)
  T* tab = reinterpret_cast<T*>(smem_raw);
  T* ybuf = tab + ((a.tab_total + 1) & ~1);
  T* fsb = ybuf + (size_t)TL * a.LS;
  T* cin = fsb + (STAGED ? (size_t)TL * a.FS : 0);
  T* cinb = cin + (size_t)P * TL * 2;
  double* bcs = reinterpret_cast<double*>(cinb + (size_t)P * TL * 2 + 2);
  bcs = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(bcs) + 7) & ~uintptr_t(7));

  const T* __restrict__ f = static_cast<const T*>(a.f);
  const T* tabT = static_cast<const T*>(a.tabT);
  for (int i = threadIdx.x; i < a.tab_total; i += blockDim.x) tab[i] = tabT[i];

  const int tid = threadIdx.x;
  const int l = tid % TL, c = tid / TL;
  const int64_t line0 = (int64_t)blockIdx.x * TL;
  const int64_t line = line0 + l;
  const bool valid = line < a.n_lines;
  int64_t base, st;
  if (STAGED) {
    base = line * n;
    st = 1;
  } else {
    int64_t o = line / a.inner, i = line % a.inner;
    base = o * (int64_t)n * a.inner + i;
    st = a.inner;
  }
  if (STAGED) {
    // coalesced copy of TL contiguous lines into padded rows of fs
    int64_t nl = min((int64_t)TL, a.n_lines - line0);
    int64_t cnt = nl * n;
    const T* src = f + line0 * n;
    for (int64_t e = tid; e < cnt; e += blockDim.x) {
      int ll = (int)(e / n), k = (int)(e % n);
      fsb[ll * a.FS + k] = src[e];
    }
    for (int64_t e = cnt + tid; e < (int64_t)TL * n; e += blockDim.x) {
      int ll = (int)(e / n), k = (int)(e % n);
      fsb[ll * a.FS + k] = T(0);
    }
  }
  __syncthreads();
  const T* fs = STAGED ? fsb + l * a.FS : nullptr;
  T* yl = ybuf + (size_t)l * a.LS;  // this line's (y0,y1) pairs

  const int j0 = c * C;
  const int j1 = min(j0 + C, n_rows);
  const T c1 = tab[lay.bc() + 30], c2 = tab[lay.bc() + 31];
  const T* Lfi = tab + lay.cst();
  const T* Pi = Lfi + 4;
  const T* Hi = Lfi + 8;
  const T* Plast = Lfi + 12;

  // ---- boundary closures (FP64) -------------------------------------------
  if (!PERIODIC) {
    const double* tb = a.tab + lay.bc();
    if (c == 0) {
      double r0, r1;
      if (a.ovl) { r0 = a.bcl0; r1 = a.bcl1; }
      else {
        double fv[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) fv[k] = (double)load_f<T, STAGED>(f, fs, base, st, k, valid);
        r0 = tb[16] * fv[0] + tb[17] * fv[1] + tb[18] * fv[2] + tb[19] * fv[3];
        r1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
      }
      bcs[l * 4 + 0] = r0;
      bcs[l * 4 + 1] = r1;
    }
    if (c == P - 1) {
      double r0, r1;
      if (a.ovr) { r0 = a.bcr0; r1 = a.bcr1; }
      else {
        double fv[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) fv[k] = (double)load_f<T, STAGED>(f, fs, base, st, n - 1 - k, valid);
        r0 = tb[20] * fv[0] + tb[21] * fv[1] + tb[22] * fv[2] + tb[23] * fv[3];
        r1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
      }
      bcs[l * 4 + 2] = r0;
      bcs[l * 4 + 3] = r1;
    }
  }
  __syncthreads();

  // ---- forward local sweep: y_j = b_j - Lf_j y_{j-1} (zero carry-in) -------
  {
    const int Nn = n - 1;  // periodic: number of unique nodes
    auto node = [&](int k) -> int {
      if (PERIODIC) { if (k < 0) return k + Nn; if (k >= Nn) return k - Nn; }
      return k;
    };
    // row j <-> node k = j+1 (wall) or j (periodic)
    const int off = PERIODIC ? 0 : 1;
    T fm = T(0), f0 = T(0);
    if (j0 < j1) {
      fm = load_f<T, STAGED>(f, fs, base, st, node(j0 + off - 1), valid);
      f0 = load_f<T, STAGED>(f, fs, base, st, node(j0 + off), valid);
    }
    V2<T> y{T(0), T(0)};
    for (int j = j0; j < j1; ++j) {
      T fp = load_f<T, STAGED>(f, fs, base, st, node(j + off + 1), valid);
      V2<T> b{c1 * (fp - fm), c2 * ((fm - T(2) * f0) + fp)};
      if (!PERIODIC) {
        if (j == 0) {
          const double* tb = a.tab + lay.bc();
          double l0 = bcs[l * 4 + 0], l1 = bcs[l * 4 + 1];
          double s0 = tb[0] * l0 + tb[1] * l1, s1 = tb[2] * l0 + tb[3] * l1;
          b.a = (T)((double)b.a - s0);
          b.b = (T)((double)b.b - s1);
        }
        if (j == n_rows - 1) {
          const double* tb = a.tab + lay.bc();
          double r0 = bcs[l * 4 + 2], r1 = bcs[l * 4 + 3];
          double s0 = tb[4] * r0 + tb[5] * r1, s1 = tb[6] * r0 + tb[7] * r1;
          b.a = (T)((double)b.a - s0);
          b.b = (T)((double)b.b - s1);
        }
      }
      if (j == j0) {
        y = b;
      } else {
        const T* Lf = (!PERIODIC && c == 0) ? tab + lay.lf0() + 4 * j : Lfi;
        V2<T> t = mv(Lf, y);
        y = {b.a - t.a, b.b - t.b};
      }
      yl[2 * j] = y.a;
      yl[2 * j + 1] = y.b;
      fm = f0;
      f0 = fp;
    }
  }
  __syncthreads();

  // ---- forward carry scan (one thread per line) ----------------------------
  T* cinl = cin + (size_t)l * P * 2;
  if (c == 0) {
    const T* Phi = tab + lay.phi();
    if (!PERIODIC) {
      int e0 = min(C, n_rows) - 1;
      V2<T> Y{yl[2 * e0], yl[2 * e0 + 1]};
      for (int cc = 1; cc < P; ++cc) {
        cinl[2 * cc] = Y.a;
        cinl[2 * cc + 1] = Y.b;
        int s = cc * C, e = min(s + C, n_rows);
        V2<T> t = mv(Phi + 4 * (e - s - 1), Y);
        Y = {yl[2 * (e - 1)] + t.a, yl[2 * (e - 1) + 1] + t.b};
      }
    } else {
      V2<T> Y{T(0), T(0)};
      for (int cc = 0; cc < P; ++cc) {
        int s = cc * C, e = min(s + C, n_rows);
        V2<T> t = mv(Phi + 4 * (e - s - 1), Y);
        Y = {yl[2 * (e - 1)] + t.a, yl[2 * (e - 1) + 1] + t.b};
      }
      Y = mv(Lfi + 16, Y);  // Gf = (I - T_ring)^-1
      for (int cc = 0; cc < P; ++cc) {
        cinl[2 * cc] = Y.a;
        cinl[2 * cc + 1] = Y.b;
        int s = cc * C, e = min(s + C, n_rows);
        V2<T> t = mv(Phi + 4 * (e - s - 1), Y);
        Y = {yl[2 * (e - 1)] + t.a, yl[2 * (e - 1) + 1] + t.b};
      }
    }
  }
  __syncthreads();

  // ---- forward fix-up + backward local sweep --------------------------------
  {
    const bool has_cin = PERIODIC || c > 0;
    V2<T> Yin{T(0), T(0)};
    if (has_cin) { Yin.a = cinl[2 * c]; Yin.b = cinl[2 * c + 1]; }
    const T* Phi = tab + lay.phi();
    if (has_cin) {
      for (int j = j0; j < j1; ++j) {
        V2<T> t = mv(Phi + 4 * (j - j0), Yin);
        yl[2 * j] += t.a;
        yl[2 * j + 1] += t.b;
      }
    }
    V2<T> xn{T(0), T(0)};
    for (int j = j1 - 1; j >= j0; --j) {
      V2<T> y{yl[2 * j], yl[2 * j + 1]};
      V2<T> x;
      if (!PERIODIC && c == 0) {
        V2<T> p = mv(tab + lay.p0() + 4 * j, y);
        V2<T> q = mv(tab + lay.h0() + 4 * j, xn);
        x = {p.a - q.a, p.b - q.b};
      } else if (!PERIODIC && j == n_rows - 1) {
        x = mv(Plast, y);
      } else {
        V2<T> p = mv(Pi, y);
        V2<T> q = mv(Hi, xn);
        x = {p.a - q.a, p.b - q.b};
      }
      yl[2 * j] = x.a;
      yl[2 * j + 1] = x.b;
      xn = x;
    }
  }
  __syncthreads();

  // ---- backward carry scan --------------------------------------------------
  T* cinbl = cinb + (size_t)l * P * 2;
  if (c == 0) {
    const T* Psi = tab + lay.psi();
    if (!PERIODIC) {
      int s = (P - 1) * C;
      V2<T> X{yl[2 * s], yl[2 * s + 1]};
      for (int cc = P - 2; cc >= 0; --cc) {
        cinbl[2 * cc] = X.a;
        cinbl[2 * cc + 1] = X.b;
        if (cc >= 1) {
          int s2 = cc * C;
          V2<T> t = mv(Psi + 4 * C, X);
          X = {yl[2 * s2] + t.a, yl[2 * s2 + 1] + t.b};
        }
      }
    } else {
      V2<T> X{T(0), T(0)};
      for (int cc = P - 1; cc >= 0; --cc) {
        int s = cc * C, e = min(s + C, n_rows);
        V2<T> t = mv(Psi + 4 * (e - s), X);
        X = {yl[2 * s] + t.a, yl[2 * s + 1] + t.b};
      }
      X = mv(Lfi + 20, X);  // Gb = (I - R_ring)^-1
      for (int cc = P - 1; cc >= 0; --cc) {
        cinbl[2 * cc] = X.a;
        cinbl[2 * cc + 1] = X.b;
        int s = cc * C, e = min(s + C, n_rows);
        V2<T> t = mv(Psi + 4 * (e - s), X);
        X = {yl[2 * s] + t.a, yl[2 * s + 1] + t.b};
      }
    }
  }
  __syncthreads();

  // ---- backward fix-up (+ direct output for strided axes) ------------------
  const double* J = a.J;
  T* d1 = static_cast<T*>(a.d1);
  T* d2 = static_cast<T*>(a.d2);
  {
    const bool has_cin = PERIODIC || c < P - 1;
    V2<T> Xin{T(0), T(0)};
    if (has_cin) { Xin.a = cinbl[2 * c]; Xin.b = cinbl[2 * c + 1]; }
    const T* Psi = tab + lay.psi();
    for (int j = j0; j < j1; ++j) {
      V2<T> x{yl[2 * j], yl[2 * j + 1]};
      if (has_cin) {
        const T* m = (!PERIODIC && c == 0) ? tab + lay.psi0() + 4 * j : Psi + 4 * (j1 - j);
        V2<T> t = mv(m, Xin);
        x.a += t.a;
        x.b += t.b;
        yl[2 * j] = x.a;
        yl[2 * j + 1] = x.b;
      }
      if (!STAGED && valid) {
        int k = PERIODIC ? j : j + 1;
        T o1 = x.a, o2 = x.b;
        if (J) {
          double Jk = J[k], dJk = J[n + k];
          o1 = (T)(Jk * (double)x.a);
          o2 = (T)(Jk * Jk * (double)x.b + Jk * dJk * (double)x.a);
        }
        if (d1) d1[base + (int64_t)k * st] = o1;
        if (d2) d2[base + (int64_t)k * st] = o2;
      }
    }
  }
  __syncthreads();

  // ---- boundary nodes / staged output ---------------------------------------
  auto boundary_pair = [&](int ll, bool left, double& o1, double& o2) {
    const double* tb = a.tab + lay.bc();
    const T* yy = ybuf + (size_t)ll * a.LS;
    if (left) {
      double x0 = (double)yy[0], x1 = (double)yy[1];
      o1 = (tb[8] * x0 + tb[9] * x1) + bcs[ll * 4 + 0];
      o2 = (tb[10] * x0 + tb[11] * x1) + bcs[ll * 4 + 1];
    } else {
      int jl = n_rows - 1;
      double x0 = (double)yy[2 * jl], x1 = (double)yy[2 * jl + 1];
      o1 = (tb[12] * x0 + tb[13] * x1) + bcs[ll * 4 + 2];
      o2 = (tb[14] * x0 + tb[15] * x1) + bcs[ll * 4 + 3];
    }
  };
  auto metric = [&](int k, double& o1, double& o2) {
    if (J) {
      double Jk = J[k], dJk = J[n + k];
      double t1 = Jk * o1;
      o2 = Jk * Jk * o2 + Jk * dJk * o1;
      o1 = t1;
    }
  };
  if (!STAGED) {
    if (valid) {
      if (!PERIODIC) {
        if (c == 0) {
          double o1, o2;
          boundary_pair(l, true, o1, o2);
          metric(0, o1, o2);
          if (d1) d1[base] = (T)o1;
          if (d2) d2[base] = (T)o2;
        }
        if (c == P - 1) {
          double o1, o2;
          boundary_pair(l, false, o1, o2);
          metric(n - 1, o1, o2);
          if (d1) d1[base + (int64_t)(n - 1) * st] = (T)o1;
          if (d2) d2[base + (int64_t)(n - 1) * st] = (T)o2;
        }
      } else if (c == 0) {
        double o1 = (double)yl[0], o2 = (double)yl[1];
        metric(n - 1, o1, o2);
        if (d1) d1[base + (int64_t)(n - 1) * st] = (T)o1;
        if (d2) d2[base + (int64_t)(n - 1) * st] = (T)o2;
      }
    }
  } else {
    // coalesced write of TL contiguous lines
    int64_t nl = min((int64_t)TL, a.n_lines - line0);
    int64_t cnt = nl * n;
    for (int64_t e = tid; e < cnt; e += blockDim.x) {
      int ll = (int)(e / n), k = (int)(e % n);
      const T* yy = ybuf + (size_t)ll * a.LS;
      double o1, o2;
      if (!PERIODIC) {
        if (k == 0) boundary_pair(ll, true, o1, o2);
        else if (k == n - 1) boundary_pair(ll, false, o1, o2);
        else { o1 = (double)yy[2 * (k - 1)]; o2 = (double)yy[2 * (k - 1) + 1]; }
      } else {
        int kk = (k == n - 1) ? 0 : k;
        o1 = (double)yy[2 * kk];
        o2 = (double)yy[2 * kk + 1];
      }
      if (J) metric(k, o1, o2);
      if (d1) d1[line0 * n + e] = (T)o1;
      if (d2) d2[line0 * n + e] = (T)o2;
    }
  }
}

template <typename T>
__global__ void wall_zero_kernel(T* g, int64_t outer, int64_t n, int64_t inner) {
  int64_t tot = outer * inner * 2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t side = e / (outer * inner), r = e % (outer * inner);
    int64_t o = r / inner, i = r % inner;
    int64_t k = side ? n - 1 : 0;
    g[o * n * inner + k * inner + i] = T(0);
  }
}

// ---- host: factor tables ---------------------------------------------------

int build_tables(tpf_ccd_plan* p, std::vector<double>& tab) {
  const double h = p->h;
  const int n_rows = p->n_rows;
  const M2 L = {kAlpha1, kB1 * h, kB2 / h, kBeta2};
  const M2 U = {kAlpha1, -kB1 * h, -kB2 / h, kBeta2};
  const M2 Ml = {-1.5, 1.5 * h, 0.0, 0.0};
  const M2 Mr = {-1.5, -1.5 * h, 0.0, 0.0};
  // fixed point of LU = I - L LU^-1 U (interior block LU factor)
  M2 LUi = eye();
  for (int it = 0; it < 400; ++it) LUi = sub(eye(), mul(mul(L, inv(LUi)), U));
  const M2 Pinf = inv(LUi), Lfinf = mul(L, Pinf), Hinf = mul(Pinf, U);

  int C = p->C;
  for (;;) {
    TabLayout lay{C};
    tab.assign(lay.total(), 0.0);
    bool converged = true;
    if (p->bc == TPF_BC_WALL) {
      // per-row factors of the folded system (ccd_solver_helpers.py:238-245)
      std::vector<M2> LU(n_rows), Lf(n_rows), Pm(n_rows), Hm(n_rows);
      for (int j = 0; j < n_rows; ++j) {
        M2 D = eye();
        if (j == 0) D = add(D, mul(L, Ml));
        if (j == n_rows - 1) D = add(D, mul(U, Mr));
        if (j == 0) {
          LU[j] = D;
          Lf[j] = {0, 0, 0, 0};
        } else {
          Lf[j] = mul(L, inv(LU[j - 1]));
          LU[j] = sub(D, mul(Lf[j], U));
        }
        double dt = det(LU[j]);
        if (!std::isfinite(dt) || std::fabs(dt) < 1e-300) {
          tpf::set_error("CCD block-tridiagonal factorization encountered a singular pivot at block %d", j);
          return TPF_ESINGULAR;
        }
        Pm[j] = inv(LU[j]);
        Hm[j] = (j < n_rows - 1) ? mul(Pm[j], U) : M2{0, 0, 0, 0};
      }
      // rows >= C (except the last) must sit at the fixed point
      for (int j = C; j < n_rows - 1; ++j) {
        double e = std::max(maxabs(sub(Lf[j], Lfinf)) / maxabs(Lfinf),
                            std::max(maxabs(sub(Pm[j], Pinf)) / maxabs(Pinf),
                                     maxabs(sub(Hm[j], Hinf)) / maxabs(Hinf)));
        if (!(e < 1e-14)) { converged = false; break; }
      }
      if (!converged) {
        if (C >= 256) { tpf::set_error("CCD factor recurrence did not converge"); return TPF_ESINGULAR; }
        C *= 2;
        continue;
      }
      int c0 = std::min(C, n_rows);
      for (int j = 0; j < c0; ++j) {
        for (int q = 0; q < 4; ++q) {
          tab[lay.lf0() + 4 * j + q] = Lf[j][q];
          tab[lay.p0() + 4 * j + q] = Pm[j][q];
          tab[lay.h0() + 4 * j + q] = Hm[j][q];
        }
      }
      // Psi0_j = prod_{m=j}^{c0-1} (-H_m): dependence of chunk-0 x_j on x_{c0}
      M2 acc = eye();
      for (int j = c0 - 1; j >= 0; --j) {
        acc = mul(neg(Hm[j]), acc);
        for (int q = 0; q < 4; ++q) tab[lay.psi0() + 4 * j + q] = acc[q];
      }
      M2 pl = Pm[n_rows - 1];
      for (int q = 0; q < 4; ++q) tab[lay.cst() + 12 + q] = pl[q];
    }
    // Phi_k = (-Lf)^(k+1), Psi_k = (-H)^k
    M2 acc = eye();
    for (int k = 0; k < C; ++k) {
      acc = mul(neg(Lfinf), acc);
      for (int q = 0; q < 4; ++q) tab[lay.phi() + 4 * k + q] = acc[q];
    }
    acc = eye();
    for (int k = 0; k <= C; ++k) {
      for (int q = 0; q < 4; ++q) tab[lay.psi() + 4 * k + q] = acc[q];
      acc = mul(neg(Hinf), acc);
    }
    for (int q = 0; q < 4; ++q) {
      tab[lay.cst() + q] = Lfinf[q];
      tab[lay.cst() + 4 + q] = Pinf[q];
      tab[lay.cst() + 8 + q] = Hinf[q];
    }
    if (p->bc == TPF_BC_PERIODIC) {
      // ring transfers of the two cyclic recurrences
      const int P = (n_rows + C - 1) / C;
      M2 Tr = eye(), Rr = eye();
      for (int cc = 0; cc < P; ++cc) {
        int s = cc * C, e = std::min(s + C, n_rows);
        M2 Tc, Rc;
        for (int q = 0; q < 4; ++q) {
          Tc[q] = tab[lay.phi() + 4 * (e - s - 1) + q];
          Rc[q] = tab[lay.psi() + 4 * (e - s) + q];
        }
        Tr = mul(Tc, Tr);   // T_{P-1} ... T_0
        Rr = mul(Rr, Rc);   // R_0 R_1 ... R_{P-1}
      }
      M2 Gf = inv(sub(eye(), Tr)), Gb = inv(sub(eye(), Rr));
      for (int q = 0; q < 4; ++q) {
        tab[lay.cst() + 16 + q] = Gf[q];
        tab[lay.cst() + 20 + q] = Gb[q];
      }
    }
    // closure constants
    const int b = lay.bc();
    const M2 L0 = L, UN = U;
    for (int q = 0; q < 4; ++q) {
      tab[b + q] = L0[q];
      tab[b + 4 + q] = UN[q];
      tab[b + 8 + q] = Ml[q];
      tab[b + 12 + q] = Mr[q];
    }
    const double cIl[4] = {-23.0 / 6.0, 21.0 / 4.0, -1.5, 1.0 / 12.0};
    const double cII[6] = {45.0, -154.0, 214.0, -156.0, 61.0, -10.0};
    for (int q = 0; q < 4; ++q) {
      tab[b + 16 + q] = cIl[q] / h;
      tab[b + 20 + q] = -cIl[q] / h;
    }
    for (int q = 0; q < 6; ++q) tab[b + 24 + q] = cII[q] / (12.0 * h * h);
    tab[b + 30] = kA1 / h;
    tab[b + 31] = kA2 / (h * h);
    p->C = C;
    p->P = (n_rows + C - 1) / C;
    return TPF_OK;
  }
}

struct LaunchShape {
  int TL, LS, FS;
  size_t smem;
};

template <typename T>
LaunchShape pick_shape(const tpf_ccd_plan* p, bool staged, int64_t n_lines) {
  TabLayout lay{p->C};
  const int n = (int)p->n_pts;
  const int LS = 2 * p->n_rows + 1;
  const int FS = (n % 2) ? n : n + 1;
  int best = -1;
  LaunchShape s{};
  const int tl_opts[3] = {32, 16, 8};
  for (int t = 0; t < 3; ++t) {
    int TL = tl_opts[t];
    if (TL * p->P > 512) continue;
    size_t sm = sizeof(T) * (((size_t)lay.total() + 1) & ~(size_t)1) + sizeof(T) * (size_t)TL * LS +
                (staged ? sizeof(T) * (size_t)TL * FS : 0) + sizeof(T) * (size_t)p->P * TL * 4 +
                2 * sizeof(T) + 16 + sizeof(double) * TL * 4;
    if (sm > 220 * 1024) continue;
    // prefer >= 2 CTAs per SM, then more lines per CTA; few lines -> small TL
    int score = (sm <= 110 * 1024 ? 100 : 0) + TL;
    if (n_lines < (int64_t)TL * 148 && TL > 8) score -= 50;
    if (score > best) { best = score; s = {TL, LS, FS, sm}; }
  }
  if (best < 0) s.TL = 0;
  return s;
}

template <typename T>
int launch_ccd(const tpf_ccd_plan* p, int64_t outer, int64_t inner, const void* f, void* d1, void* d2,
               const double* bcl, const double* bcr, int flags, cudaStream_t stream) {
  const bool staged = (inner == 1);
  const int64_t n_lines = outer * inner;
  if (n_lines == 0) return TPF_OK;
  LaunchShape s = pick_shape<T>(p, staged, n_lines);
  TPF_CHECK_ARG(s.TL > 0, "CCD axis of %lld points does not fit the line kernel's shared memory",
                (long long)p->n_pts);
  CcdArgs a{};
  a.f = f; a.d1 = d1; a.d2 = d2;
  a.outer = outer; a.inner = inner; a.n_lines = n_lines;
  a.n = (int)p->n_pts; a.n_rows = p->n_rows; a.C = p->C; a.P = p->P; a.TL = s.TL;
  a.LS = s.LS; a.FS = s.FS;
  a.tab_total = TabLayout{p->C}.total();
  a.tab = p->d_tab;
  a.tabT = std::is_same<T, double>::value ? (const void*)p->d_tab : (const void*)p->d_tabf;
  a.J = ((flags & TPF_CCD_APPLY_METRIC) && p->has_metric) ? p->d_J : nullptr;
  a.ovl = bcl ? 1 : 0;
  a.ovr = bcr ? 1 : 0;
  if (bcl) { a.bcl0 = bcl[0]; a.bcl1 = bcl[1]; }
  if (bcr) { a.bcr0 = bcr[0]; a.bcr1 = bcr[1]; }
  dim3 grid((unsigned)((n_lines + s.TL - 1) / s.TL)), block(s.TL * p->P);
  const bool per = (p->bc == TPF_BC_PERIODIC) && !a.ovl && !a.ovr;
  void (*kern)(CcdArgs);
  if (per) kern = staged ? ccd_line_kernel<T, true, true> : ccd_line_kernel<T, true, false>;
  else kern = staged ? ccd_line_kernel<T, false, true> : ccd_line_kernel<T, false, false>;
  TPF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem));
  kern<<<grid, block, s.smem, stream>>>(a);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

}  // namespace

extern "C" {

int tpf_ccd_plan_create(tpf_ccd_plan** out, int64_t n_pts, double h, int bc, int dtype) {
  TPF_CHECK_ARG(out != nullptr, "plan pointer is NULL");
  *out = nullptr;
  TPF_CHECK_ARG(bc == TPF_BC_WALL || bc == TPF_BC_PERIODIC, "unsupported boundary type %d", bc);
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "unsupported dtype %d", dtype);
  TPF_CHECK_ARG(std::isfinite(h) && h > 0.0, "grid spacing must be positive and finite");
  if (bc == TPF_BC_WALL) {
    TPF_CHECK_ARG(n_pts >= 6,
                  "CCD wall Eq-II boundary closure requires n_pts >= 6 for the six-point O(h^4) formula");
  } else {
    TPF_CHECK_ARG(n_pts >= 4, "Need >= 3 unique nodes for periodic CCD; got %lld", (long long)(n_pts - 1));
  }
  TPF_CHECK_ARG(n_pts <= 8193, "CCD axis longer than 8193 points is not supported");
  auto* p = new tpf_ccd_plan();
  p->n_pts = n_pts;
  p->h = h;
  p->bc = bc;
  p->dtype = dtype;
  p->n_rows = (bc == TPF_BC_WALL) ? (int)(n_pts - 2) : (int)(n_pts - 1);
  p->C = std::max(32, (p->n_rows + 31) / 32);
  std::vector<double> tab;
  int st = build_tables(p, tab);
  if (st != TPF_OK) { delete p; return st; }
  if (cudaMalloc(&p->d_tab, tab.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&p->d_tabf, tab.size() * sizeof(float)) != cudaSuccess) {
    tpf::set_error("cudaMalloc of CCD tables failed");
    cudaFree(p->d_tab);
    delete p;
    return TPF_ECUDA;
  }
  std::vector<float> tf(tab.begin(), tab.end());
  if (cudaMemcpy(p->d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_tabf, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    tpf::set_error("copy of CCD tables failed");
    cudaFree(p->d_tab);
    cudaFree(p->d_tabf);
    delete p;
    return TPF_ECUDA;
  }
  *out = p;
  return TPF_OK;
}

int tpf_ccd_plan_destroy(tpf_ccd_plan* p) {
  if (!p) return TPF_OK;
  cudaFree(p->d_tab);
  cudaFree(p->d_tabf);
  cudaFree(p->d_J);
  delete p;
  return TPF_OK;
}

int tpf_ccd_plan_set_metric(tpf_ccd_plan* p, const double* J, const double* dJ) {
  TPF_CHECK_ARG(p && J && dJ, "NULL argument");
  if (!p->d_J) TPF_CUDA_TRY(cudaMalloc(&p->d_J, 2 * p->n_pts * sizeof(double)));
  TPF_CUDA_TRY(cudaMemcpy(p->d_J, J, p->n_pts * sizeof(double), cudaMemcpyHostToDevice));
  TPF_CUDA_TRY(cudaMemcpy(p->d_J + p->n_pts, dJ, p->n_pts * sizeof(double), cudaMemcpyHostToDevice));
  p->has_metric = true;
  return TPF_OK;
}

int tpf_ccd_apply(const tpf_ccd_plan* p, int64_t outer, int64_t inner, const void* f, void* d1, void* d2,
                  const double* bc_left, const double* bc_right, int flags, void* stream) {
  TPF_CHECK_ARG(p != nullptr, "plan is NULL");
  TPF_CHECK_ARG(outer >= 0 && inner >= 1, "invalid line decomposition outer=%lld inner=%lld",
                (long long)outer, (long long)inner);
  TPF_CHECK_ARG(f != nullptr, "input is NULL");
  TPF_CHECK_ARG(d1 != nullptr || d2 != nullptr, "no output requested");
  TPF_CHECK_ARG(!(flags & TPF_CCD_APPLY_METRIC) || p->has_metric, "metric requested but not set");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->dtype == TPF_F64) return launch_ccd<double>(p, outer, inner, f, d1, d2, bc_left, bc_right, flags, s);
  return launch_ccd<float>(p, outer, inner, f, d1, d2, bc_left, bc_right, flags, s);
}

int tpf_ccd_enforce_wall_neumann(const tpf_ccd_plan* p, int64_t outer, int64_t inner, void* grad,
                                 void* stream) {
  TPF_CHECK_ARG(p != nullptr && grad != nullptr, "NULL argument");
  if (p->bc != TPF_BC_WALL || outer * inner == 0) return TPF_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t tot = outer * inner * 2;
  int blocks = (int)std::min<int64_t>((tot + 255) / 256, 4096);
  if (p->dtype == TPF_F64)
    wall_zero_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double*>(grad), outer, p->n_pts, inner);
  else
    wall_zero_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float*>(grad), outer, p->n_pts, inner);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

}  // extern "C"

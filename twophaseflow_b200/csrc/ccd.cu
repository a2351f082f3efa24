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
#include <map>

struct LaneShape_ {
  int warps, nbuf, max_bps;
};

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

// Table layout (doubles).  C = chunk length, H0 = rows [0, H0) of the wall
// "head" that carry per-row factors (the block-LU factors only reach the
// fixed point ~30 rows away from the wall closure).
struct TabLayout {
  int C, H0;
  __host__ __device__ int head() const { return 0; }                // H0 x 20: Lf P H PhiH PsiH
  __host__ __device__ int phi() const { return 20 * H0; }           // C x 4
  __host__ __device__ int psi() const { return 20 * H0 + 4 * C; }   // (C+1) x 4
  __host__ __device__ int cst() const { return 20 * H0 + 8 * C + 4; }  // Lfi Pi Hi Plast Gf Gb
  __host__ __device__ int bc() const { return cst() + 24; }         // L0 UN Ml Mr cIl cIr cII(6) c1 c2
  __host__ __device__ int total() const { return bc() + 32; }
};

}  // namespace

struct tpf_ccd_plan {
  int64_t n_pts = 0;
  double h = 0.0;
  int bc = TPF_BC_WALL;
  int dtype = TPF_F64;
  int n_rows = 0, C = 32, P = 1, H0 = 0;
  double* d_tab = nullptr;   // double table
  float* d_tabf = nullptr;   // float copy (interior factors for F32)
  double* d_J = nullptr;     // metric J, dJ (n_pts each)
  bool has_metric = false;
  // lane-per-line kernel table (factors, ring closures, head rows)
  double* d_ltab = nullptr;
  float* d_ltabf = nullptr;
  int ltab_total = 0;
  std::vector<double> ltab_host;
  // lane-kernel launch shapes picked by the autotuner, per call signature
  mutable std::map<uint64_t, LaneShape_> lane_tuned;
  bool autotune = true;
  // FP32 per-row block-LU factors of the folded wall system (Lf, P, H per
  // row) for the iterative-refinement correction solves, built on first use
  mutable float* d_rfac = nullptr;
};

namespace {

struct CcdArgs {
  const void* f;
  void* d1;
  void* d2;
  int64_t outer, inner, n_lines;
  int n, n_rows, C, P, H0, TL, tl_shift;
  int LS, FS;             // ybuf line stride / staged-f line stride (elements)
  int nbuf;               // f tile buffers (1 or 2)
  int n_tiles;
  int tab_total;
  const double* tab;      // double table (closures)
  const void* tabT;       // table in compute type
  const double* J;        // metric (J[0..n), dJ[n..2n)) or nullptr
  int ovl, ovr;           // wall closure overrides (left / right)
  double bcl0, bcl1, bcr0, bcr1;
  // variable-density epilogue: out (+)= d2/rho - (drho/rho^2) d1 instead of d1, d2
  const void* vd_rho;
  const void* vd_drho;
  void* vd_out;
  int vd_accumulate;
  // velocity-corrector epilogue: out = u* - (dt / rho) d1 instead of d1, d2;
  // on wall planes (first / last node of a line) d1 counts as 0, so out = u*
  const void* cr_u;
  const void* cr_rho;
  void* cr_out;
  double cr_dt;
  int cr_wall;
};

template <typename T>
struct V2 { T a, b; };

// Write one node's result: either (d1, d2) or the variable-density term.
template <typename T>
__device__ __forceinline__ void store_out(const CcdArgs& a, int64_t gi, double o1, double o2, int k) {
  if (a.cr_out) {
    // u_new = u* - (dt / rho) dp/dx, with the reference's operation order
    // (quotient, product, difference; no fused multiply-add).  The loads are
    // read-only-path loads so that they need not wait for earlier nodes'
    // stores: every address is read once, by the lane that later writes it
    // (u_out may be u_star), so no stale value can be read.
    const double u = (double)__ldg(static_cast<const T*>(a.cr_u) + gi);
    double v = u;
    if (!(a.cr_wall && (k == 0 || k == a.n - 1))) {   // k: node along the line
      const double q = a.cr_dt / (double)__ldg(static_cast<const T*>(a.cr_rho) + gi);
      v = __dsub_rn(u, __dmul_rn(q, o1));
    }
    static_cast<T*>(a.cr_out)[gi] = (T)v;
    return;
  }
  if (a.vd_out) {
    const double r = (double)static_cast<const T*>(a.vd_rho)[gi];
    const double dr = (double)static_cast<const T*>(a.vd_drho)[gi];
    double t = o2 / r - (dr / (r * r)) * o1;
    T* out = static_cast<T*>(a.vd_out);
    if (a.vd_accumulate) t = (double)out[gi] + t;
    out[gi] = (T)t;
    return;
  }
  if (a.d1) static_cast<T*>(a.d1)[gi] = (T)o1;
  if (a.d2) static_cast<T*>(a.d2)[gi] = (T)o2;
}

template <typename T>
__device__ __forceinline__ V2<T> mv(const T* m, V2<T> v) {
  return {m[0] * v.a + m[1] * v.b, m[2] * v.a + m[3] * v.b};
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
  unsigned int sa = (unsigned int)__cvta_generic_to_shared(smem);
  int src = valid ? BYTES : 0;   // src-size 0 -> zero fill
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gmem), "n"(BYTES), "r"(src)
               : "memory");
}
// cp.async with an L2 eviction-priority policy (createpolicy), for staging
// copies whose lines are re-read later (evict_last) or read for the last
// time (evict_first)
template <int BYTES>
__device__ __forceinline__ void cp_async_pol(void* smem, const void* gmem, uint64_t pol) {
  unsigned int sa = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], %2, %2, %3;\n" ::"r"(sa), "l"(gmem), "n"(BYTES),
               "l"(pol)
               : "memory");
}
__device__ __forceinline__ uint64_t pol_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t pol_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Stage a read-only table into shared memory with asynchronous copies: every
// thread issues its share and waits once, so the copy costs one global round
// trip rather than one per element a thread copies (a block of one warp and a
// 700-entry table otherwise spends ~10 us here, longer than a small field's
// whole solve).  Called before any other asynchronous copy of the block.
template <typename T>
__device__ __forceinline__ void stage_table(T* dst, const T* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) cp_async<sizeof(T)>(dst + i, src + i, true);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
}

// Issue the asynchronous copy of tile `t` (TL lines x n points) into fb.
// Strided axis: fb[k*TL + l]; contiguous axis: fb[l*FS + k].  lb receives the
// global base offset of each line (strided) for the output pass.
template <typename T, bool CONTIG>
__device__ __forceinline__ void issue_tile(const CcdArgs& a, const T* __restrict__ f, T* fb, long long* lb, int t) {
  const int TL = a.TL, n = a.n;
  const int64_t line0 = (int64_t)t * TL;
  if (CONTIG) {
    const int64_t nl = min((int64_t)TL, a.n_lines - line0);
    const T* src = f + line0 * n;
    const int total = TL * n;
    int l = threadIdx.x / n, k = threadIdx.x - (threadIdx.x / n) * n;
    const int step_l = blockDim.x / n, step_k = blockDim.x - step_l * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const bool v = l < nl;
      cp_async<sizeof(T)>(fb + l * a.FS + k, v ? src + e : f, v);
      l += step_l;
      k += step_k;
      if (k >= n) { k -= n; ++l; }
    }
  } else {
    if (threadIdx.x < TL) {
      const int64_t line = line0 + threadIdx.x;
      long long b = -1;
      if (line < a.n_lines) {
        const int64_t o = line / a.inner, i = line - o * a.inner;
        b = o * (int64_t)n * a.inner + i;
      }
      lb[threadIdx.x] = b;
    }
    __syncthreads();
    const int total = TL * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int k = e >> a.tl_shift, l = e & (TL - 1);
      const long long b = lb[l];
      cp_async<sizeof(T)>(fb + e, b >= 0 ? f + b + (int64_t)k * a.inner : f, b >= 0);
    }
  }
  cp_async_commit();
}

template <typename T, bool PERIODIC, bool CONTIG>
__global__ void __launch_bounds__(512, 1) ccd_line_kernel(CcdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TL = a.TL, C = a.C, P = a.P, n = a.n, n_rows = a.n_rows, H0 = a.H0;
  const TabLayout lay{C, H0};
  const int fsz = CONTIG ? TL * a.FS : TL * n;
  // shared layout: bcs(double) | lbase(2 x TL) | tab(T) | ybuf | fbuf[nbuf] | cin | cinb
  double* bcs = reinterpret_cast<double*>(smem_raw);
  long long* lbase = reinterpret_cast<long long*>(bcs + 4 * TL);
  T* tab = reinterpret_cast<T*>(lbase + 2 * TL);
  T* ybuf = tab + ((a.tab_total + 1) & ~1);
  T* fbuf = ybuf + (((size_t)TL * a.LS + 1) & ~(size_t)1);
  T* cin = fbuf + (size_t)a.nbuf * fsz;
  T* cinb = cin + (size_t)P * TL * 2;

  const T* __restrict__ f = static_cast<const T*>(a.f);
  const T* tabT = static_cast<const T*>(a.tabT);
  stage_table<T>(tab, tabT, a.tab_total);   // the table is read below (c1, c2) and in every phase

  const int tid = threadIdx.x;
  const int l = tid & (TL - 1), c = tid >> a.tl_shift;
  const int j0 = c * C;
  const int j1 = min(j0 + C, n_rows);
  const T c1 = tab[lay.bc() + 30], c2 = tab[lay.bc() + 31];
  const T* Lfi = tab + lay.cst();
  const T* Pi = Lfi + 4;
  const T* Hi = Lfi + 8;
  const T* Plast = Lfi + 12;
  const T* Phi = tab + lay.phi();
  const T* Psi = tab + lay.psi();
  const T* head = tab + lay.head();
  const double* tb = a.tab + lay.bc();
  const double* J = a.J;
  T* yl = ybuf + (size_t)l * a.LS;
  T* cinl = cin + (size_t)l * P * 2;
  T* cinbl = cinb + (size_t)l * P * 2;

  int t = blockIdx.x;
  int buf = 0;
  if (t < a.n_tiles) issue_tile<T, CONTIG>(a, f, fbuf, lbase, t);
  for (; t < a.n_tiles; t += gridDim.x) {
    const int tn = t + gridDim.x;
    if (a.nbuf == 2 && tn < a.n_tiles) {
      issue_tile<T, CONTIG>(a, f, fbuf + (size_t)(buf ^ 1) * fsz, lbase + (buf ^ 1) * TL, tn);
      cp_async_wait<1>();
    } else {
      // single buffer: this tile's copy is issued here (the first one in the prologue)
      if (a.nbuf == 1 && t != (int)blockIdx.x) issue_tile<T, CONTIG>(a, f, fbuf, lbase, t);
      cp_async_wait<0>();
    }
    __syncthreads();
    const T* fb = fbuf + (size_t)buf * fsz;
    const long long* lb = lbase + buf * TL;
    const int64_t line0 = (int64_t)t * TL;
    const bool valid = CONTIG ? (line0 + l < a.n_lines) : (lb[l] >= 0);
    auto F = [&](int k) -> T { return CONTIG ? fb[l * a.FS + k] : fb[k * TL + l]; };

    // ---- wall closures (FP64) ---------------------------------------------
    if (!PERIODIC) {
      if (c == 0) {
        double r0, r1;
        if (a.ovl) { r0 = a.bcl0; r1 = a.bcl1; }
        else {
          double fv[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) fv[k] = (double)F(k);
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
          for (int k = 0; k < 6; ++k) fv[k] = (double)F(n - 1 - k);
          r0 = tb[20] * fv[0] + tb[21] * fv[1] + tb[22] * fv[2] + tb[23] * fv[3];
          r1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
        }
        bcs[l * 4 + 2] = r0;
        bcs[l * 4 + 3] = r1;
      }
      __syncthreads();
    }

    // ---- forward local sweep: y_j = b_j - Lf_j y_{j-1}, zero carry-in --------
    {
      const int Nn = n - 1;
      const int off = PERIODIC ? 0 : 1;
      auto node = [&](int k) -> int {
        if (PERIODIC) { if (k < 0) return k + Nn; if (k >= Nn) return k - Nn; }
        return k;
      };
      T fm = T(0), f0 = T(0);
      if (j0 < j1) {
        fm = F(node(j0 + off - 1));
        f0 = F(node(j0 + off));
      }
      V2<T> y{T(0), T(0)};
      for (int j = j0; j < j1; ++j) {
        const T fp = F(node(j + off + 1));
        V2<T> b{c1 * (fp - fm), c2 * ((fm - T(2) * f0) + fp)};
        if (!PERIODIC) {
          if (j == 0) {
            const double l0 = bcs[l * 4 + 0], l1 = bcs[l * 4 + 1];
            b.a = (T)((double)b.a - (tb[0] * l0 + tb[1] * l1));
            b.b = (T)((double)b.b - (tb[2] * l0 + tb[3] * l1));
          }
          if (j == n_rows - 1) {
            const double r0 = bcs[l * 4 + 2], r1 = bcs[l * 4 + 3];
            b.a = (T)((double)b.a - (tb[4] * r0 + tb[5] * r1));
            b.b = (T)((double)b.b - (tb[6] * r0 + tb[7] * r1));
          }
        }
        if (j == j0) {
          y = b;
        } else {
          const T* Lf = (!PERIODIC && j < H0) ? head + 20 * j : Lfi;
          const V2<T> q = mv(Lf, y);
          y = {b.a - q.a, b.b - q.b};
        }
        yl[2 * j] = y.a;
        yl[2 * j + 1] = y.b;
        fm = f0;
        f0 = fp;
      }
    }
    __syncthreads();

    // ---- forward carry scan (one thread per line) ---------------------------
    if (c == 0) {
      auto Tc = [&](int s, int e) -> const T* {
        return (!PERIODIC && e - 1 < H0) ? head + 20 * (e - 1) + 12 : Phi + 4 * (e - s - 1);
      };
      if (!PERIODIC) {
        const int e0 = min(C, n_rows) - 1;
        V2<T> Y{yl[2 * e0], yl[2 * e0 + 1]};
        for (int cc = 1; cc < P; ++cc) {
          cinl[2 * cc] = Y.a;
          cinl[2 * cc + 1] = Y.b;
          const int s = cc * C, e = min(s + C, n_rows);
          const V2<T> q = mv(Tc(s, e), Y);
          Y = {yl[2 * (e - 1)] + q.a, yl[2 * (e - 1) + 1] + q.b};
        }
      } else {
        V2<T> Y{T(0), T(0)};
        for (int cc = 0; cc < P; ++cc) {
          const int s = cc * C, e = min(s + C, n_rows);
          const V2<T> q = mv(Tc(s, e), Y);
          Y = {yl[2 * (e - 1)] + q.a, yl[2 * (e - 1) + 1] + q.b};
        }
        Y = mv(Lfi + 16, Y);  // Gf = (I - T_ring)^-1
        for (int cc = 0; cc < P; ++cc) {
          cinl[2 * cc] = Y.a;
          cinl[2 * cc + 1] = Y.b;
          const int s = cc * C, e = min(s + C, n_rows);
          const V2<T> q = mv(Tc(s, e), Y);
          Y = {yl[2 * (e - 1)] + q.a, yl[2 * (e - 1) + 1] + q.b};
        }
      }
    }
    __syncthreads();

    // ---- forward fix-up + backward local sweep -------------------------------
    {
      if (PERIODIC || c > 0) {
        const V2<T> Yin{cinl[2 * c], cinl[2 * c + 1]};
        for (int j = j0; j < j1; ++j) {
          const T* m = (!PERIODIC && j < H0) ? head + 20 * j + 12 : Phi + 4 * (j - j0);
          const V2<T> q = mv(m, Yin);
          yl[2 * j] += q.a;
          yl[2 * j + 1] += q.b;
        }
      }
      V2<T> xn{T(0), T(0)};
      for (int j = j1 - 1; j >= j0; --j) {
        const V2<T> y{yl[2 * j], yl[2 * j + 1]};
        V2<T> x;
        if (!PERIODIC && j < H0) {
          const V2<T> p = mv(head + 20 * j + 4, y);
          const V2<T> q = mv(head + 20 * j + 8, xn);
          x = {p.a - q.a, p.b - q.b};
        } else if (!PERIODIC && j == n_rows - 1) {
          x = mv(Plast, y);
        } else {
          const V2<T> p = mv(Pi, y);
          const V2<T> q = mv(Hi, xn);
          x = {p.a - q.a, p.b - q.b};
        }
        yl[2 * j] = x.a;
        yl[2 * j + 1] = x.b;
        xn = x;
      }
    }
    __syncthreads();

    // ---- backward carry scan -------------------------------------------------
    if (c == 0) {
      auto Rc = [&](int s, int e) -> const T* {
        return (!PERIODIC && s < H0) ? head + 20 * s + 16 : Psi + 4 * (e - s);
      };
      if (!PERIODIC) {
        const int s = (P - 1) * C;
        V2<T> X{yl[2 * s], yl[2 * s + 1]};
        for (int cc = P - 2; cc >= 0; --cc) {
          cinbl[2 * cc] = X.a;
          cinbl[2 * cc + 1] = X.b;
          if (cc >= 1) {
            const int s2 = cc * C, e2 = min(s2 + C, n_rows);
            const V2<T> q = mv(Rc(s2, e2), X);
            X = {yl[2 * s2] + q.a, yl[2 * s2 + 1] + q.b};
          }
        }
      } else {
        V2<T> X{T(0), T(0)};
        for (int cc = P - 1; cc >= 0; --cc) {
          const int s = cc * C, e = min(s + C, n_rows);
          const V2<T> q = mv(Rc(s, e), X);
          X = {yl[2 * s] + q.a, yl[2 * s + 1] + q.b};
        }
        X = mv(Lfi + 20, X);  // Gb = (I - R_ring)^-1
        for (int cc = P - 1; cc >= 0; --cc) {
          cinbl[2 * cc] = X.a;
          cinbl[2 * cc + 1] = X.b;
          const int s = cc * C, e = min(s + C, n_rows);
          const V2<T> q = mv(Rc(s, e), X);
          X = {yl[2 * s] + q.a, yl[2 * s + 1] + q.b};
        }
      }
    }
    __syncthreads();

    // ---- backward fix-up (+ direct output for strided axes) ----------------
    {
      const bool has_cin = PERIODIC || c < P - 1;
      V2<T> Xin{T(0), T(0)};
      if (has_cin) { Xin.a = cinbl[2 * c]; Xin.b = cinbl[2 * c + 1]; }
      const long long base = CONTIG ? 0 : lb[l];
      for (int j = j0; j < j1; ++j) {
        V2<T> x{yl[2 * j], yl[2 * j + 1]};
        if (has_cin) {
          const T* m = (!PERIODIC && j < H0) ? head + 20 * j + 16 : Psi + 4 * (j1 - j);
          const V2<T> q = mv(m, Xin);
          x.a += q.a;
          x.b += q.b;
          yl[2 * j] = x.a;
          yl[2 * j + 1] = x.b;
        }
        if (!CONTIG && valid) {
          const int k = PERIODIC ? j : j + 1;
          double o1 = (double)x.a, o2 = (double)x.b;
          if (J) {
            const double Jk = J[k], dJk = J[n + k];
            o2 = Jk * Jk * o2 + Jk * dJk * o1;
            o1 = Jk * o1;
          }
          store_out<T>(a, base + (int64_t)k * a.inner, o1, o2, k);
        }
      }
    }
    __syncthreads();

    // ---- boundary nodes / contiguous-axis output ------------------------------
    auto boundary_pair = [&](int ll, bool left, double& o1, double& o2) {
      const T* yy = ybuf + (size_t)ll * a.LS;
      if (left) {
        const double x0 = (double)yy[0], x1 = (double)yy[1];
        o1 = (tb[8] * x0 + tb[9] * x1) + bcs[ll * 4 + 0];
        o2 = (tb[10] * x0 + tb[11] * x1) + bcs[ll * 4 + 1];
      } else {
        const int jl = n_rows - 1;
        const double x0 = (double)yy[2 * jl], x1 = (double)yy[2 * jl + 1];
        o1 = (tb[12] * x0 + tb[13] * x1) + bcs[ll * 4 + 2];
        o2 = (tb[14] * x0 + tb[15] * x1) + bcs[ll * 4 + 3];
      }
    };
    auto metric = [&](int k, double& o1, double& o2) {
      if (J) {
        const double Jk = J[k], dJk = J[n + k];
        const double t1 = Jk * o1;
        o2 = Jk * Jk * o2 + Jk * dJk * o1;
        o1 = t1;
      }
    };
    if (!CONTIG) {
      if (valid) {
        const long long base = lb[l];
        if (!PERIODIC) {
          if (c == 0) {
            double o1, o2;
            boundary_pair(l, true, o1, o2);
            metric(0, o1, o2);
            store_out<T>(a, base, o1, o2, 0);
          }
          if (c == P - 1) {
            double o1, o2;
            boundary_pair(l, false, o1, o2);
            metric(n - 1, o1, o2);
            store_out<T>(a, base + (int64_t)(n - 1) * a.inner, o1, o2, n - 1);
          }
        } else if (c == 0) {
          double o1 = (double)yl[0], o2 = (double)yl[1];
          metric(n - 1, o1, o2);
          store_out<T>(a, base + (int64_t)(n - 1) * a.inner, o1, o2, n - 1);
        }
      }
    } else {
      const int64_t nl = min((int64_t)TL, a.n_lines - line0);
      const int cnt = (int)nl * n;
      int ll = tid / n, k = tid - (tid / n) * n;
      const int step_l = blockDim.x / n, step_k = blockDim.x - step_l * n;
      for (int e = tid; e < cnt; e += blockDim.x) {
        const T* yy = ybuf + (size_t)ll * a.LS;
        double o1, o2;
        if (!PERIODIC) {
          if (k == 0) boundary_pair(ll, true, o1, o2);
          else if (k == n - 1) boundary_pair(ll, false, o1, o2);
          else { o1 = (double)yy[2 * (k - 1)]; o2 = (double)yy[2 * (k - 1) + 1]; }
        } else {
          const int kk = (k == n - 1) ? 0 : k;
          o1 = (double)yy[2 * kk];
          o2 = (double)yy[2 * kk + 1];
        }
        if (J) metric(k, o1, o2);
        store_out<T>(a, line0 * n + e, o1, o2, k);
        ll += step_l;
        k += step_k;
        if (k >= n) { k -= n; ++ll; }
      }
    }
    __syncthreads();
    buf ^= (a.nbuf == 2) ? 1 : 0;
  }
  cp_async_wait<0>();
}

// ---- warp-per-line fast path ------------------------------------------------------
//
// One warp solves one line: lane q owns rows [qR, qR+R) in registers.  The
// chunk carries of the two block-Thomas sweeps are affine maps (M, v) that
// compose as (M2, v2) o (M1, v1) = (M2 M1, v2 + M2 v1); a Kogge-Stone scan of
// them over the 32 lanes (shuffles, no block barrier) gives every lane its
// exact carry.  The tile of W lines is staged in shared memory by cp.async
// (double-buffered) with one padding element per R rows, so lanes reading
// rows R apart hit distinct banks; results are staged back for coalesced stores.

template <typename T>
struct Aff { T m0, m1, m2, m3, v0, v1; };

template <typename T>
__device__ __forceinline__ Aff<T> aff_compose(const Aff<T>& hi, const Aff<T>& lo) {
  Aff<T> r;
  r.m0 = hi.m0 * lo.m0 + hi.m1 * lo.m2;
  r.m1 = hi.m0 * lo.m1 + hi.m1 * lo.m3;
  r.m2 = hi.m2 * lo.m0 + hi.m3 * lo.m2;
  r.m3 = hi.m2 * lo.m1 + hi.m3 * lo.m3;
  r.v0 = hi.v0 + hi.m0 * lo.v0 + hi.m1 * lo.v1;
  r.v1 = hi.v1 + hi.m2 * lo.v0 + hi.m3 * lo.v1;
  return r;
}

template <typename T>
__device__ __forceinline__ Aff<T> aff_shfl_up(const Aff<T>& a, int d) {
  Aff<T> r;
  r.m0 = __shfl_up_sync(0xffffffffu, a.m0, d); r.m1 = __shfl_up_sync(0xffffffffu, a.m1, d);
  r.m2 = __shfl_up_sync(0xffffffffu, a.m2, d); r.m3 = __shfl_up_sync(0xffffffffu, a.m3, d);
  r.v0 = __shfl_up_sync(0xffffffffu, a.v0, d); r.v1 = __shfl_up_sync(0xffffffffu, a.v1, d);
  return r;
}

template <typename T>
__device__ __forceinline__ Aff<T> aff_shfl_down(const Aff<T>& a, int d) {
  Aff<T> r;
  r.m0 = __shfl_down_sync(0xffffffffu, a.m0, d); r.m1 = __shfl_down_sync(0xffffffffu, a.m1, d);
  r.m2 = __shfl_down_sync(0xffffffffu, a.m2, d); r.m3 = __shfl_down_sync(0xffffffffu, a.m3, d);
  r.v0 = __shfl_down_sync(0xffffffffu, a.v0, d); r.v1 = __shfl_down_sync(0xffffffffu, a.v1, d);
  return r;
}

template <typename T>
__device__ __forceinline__ Aff<T> aff_identity() { return {T(1), T(0), T(0), T(1), T(0), T(0)}; }

// copy tile t (TL lines) into fb[l*FSP + k + k/R]
template <typename T, bool CONTIG, int R>
__device__ __forceinline__ void issue_tile_padded(const CcdArgs& a, const T* __restrict__ f, T* fb, long long* lb,
                                                  int t) {
  const int TL = a.TL, n = a.n, FSP = a.FS;
  const int64_t line0 = (int64_t)t * TL;
  if (threadIdx.x < TL) {
    const int64_t line = line0 + threadIdx.x;
    long long b = -1;
    if (line < a.n_lines) {
      if (CONTIG) b = line * n;
      else {
        const int64_t o = line / a.inner, i = line - o * a.inner;
        b = o * (int64_t)n * a.inner + i;
      }
    }
    lb[threadIdx.x] = b;
  }
  __syncthreads();
  const int total = TL * n;
  if (CONTIG) {
    // consecutive threads -> consecutive k of one line (coalesced)
    int l = threadIdx.x / n, k = threadIdx.x - (threadIdx.x / n) * n;
    const int step_l = blockDim.x / n, step_k = blockDim.x - step_l * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const long long b = lb[l];
      cp_async<sizeof(T)>(fb + l * FSP + k + k / R, b >= 0 ? f + b + k : f, b >= 0);
      l += step_l;
      k += step_k;
      if (k >= n) { k -= n; ++l; }
    }
  } else {
    // consecutive threads -> consecutive lines at one k (coalesced)
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int k = e >> a.tl_shift, l = e & (TL - 1);
      const long long b = lb[l];
      cp_async<sizeof(T)>(fb + l * FSP + k + k / R, b >= 0 ? f + b + (int64_t)k * a.inner : f, b >= 0);
    }
  }
  cp_async_commit();
}

// W warps per line: the line's rows are cut into 32 W chunks of R rows (lane
// l of warp w of the line owns chunk 32 w + l); the carry scans run within
// each warp by shuffles, then across the line's warps through shared memory.
template <typename T, bool PERIODIC, bool CONTIG, int R, int W>
__global__ void __launch_bounds__(256) ccd_warp_kernel(CcdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TL = a.TL, n = a.n, n_rows = a.n_rows, H0 = a.H0, FSP = a.FS;
  const TabLayout lay{R, H0};
  const int fsz = TL * FSP;
  // shared: lbase(2 x TL) | tab | fbuf[nbuf] | sbuf
  long long* lbase = reinterpret_cast<long long*>(smem_raw);
  T* tab = reinterpret_cast<T*>(lbase + 2 * TL);
  T* fbuf = tab + ((a.tab_total + 1) & ~1);
  T* sbuf = fbuf + (size_t)a.nbuf * fsz;

  const T* __restrict__ f = static_cast<const T*>(a.f);
  const T* tabT = static_cast<const T*>(a.tabT);
  stage_table<T>(tab, tabT, a.tab_total);

  const int lane = threadIdx.x & 31;
  const int wl = (threadIdx.x >> 5) / W;        // line of the tile owned by this warp
  const int wq = (threadIdx.x >> 5) - wl * W;   // this warp's segment of the line
  const int q = wq * 32 + lane;                 // chunk of the line owned by this lane
  const int j0 = q * R;
  const int cnt = max(0, min(R, n_rows - j0));  // rows of this lane
  __shared__ Aff<T> s_tot[8 * W];               // per line of the tile (TL <= 8): warp totals
  const T c1 = tab[lay.bc() + 30], c2 = tab[lay.bc() + 31];
  const T* Lfi = tab + lay.cst();
  const T Lf0 = Lfi[0], Lf1 = Lfi[1], Lf2 = Lfi[2], Lf3 = Lfi[3];
  const T P0 = Lfi[4], P1 = Lfi[5], P2 = Lfi[6], P3 = Lfi[7];
  const T H0m = Lfi[8], H1m = Lfi[9], H2m = Lfi[10], H3m = Lfi[11];
  const T* Plast = Lfi + 12;
  const T* Phi = tab + lay.phi();
  const T* Psi = tab + lay.psi();
  const T* head = tab + lay.head();
  const double* tb = a.tab + lay.bc();
  const double* J = a.J;
  const bool in_head = !PERIODIC && j0 < H0;

  int t = blockIdx.x;
  int buf = 0;
  if (t < a.n_tiles) issue_tile_padded<T, CONTIG, R>(a, f, fbuf, lbase, t);
  for (; t < a.n_tiles; t += gridDim.x) {
    const int tn = t + gridDim.x;
    if (a.nbuf == 2 && tn < a.n_tiles) {
      issue_tile_padded<T, CONTIG, R>(a, f, fbuf + (size_t)(buf ^ 1) * fsz, lbase + (buf ^ 1) * TL, tn);
      cp_async_wait<1>();
    } else {
      if (a.nbuf == 1 && t != (int)blockIdx.x) issue_tile_padded<T, CONTIG, R>(a, f, fbuf, lbase, t);
      cp_async_wait<0>();
    }
    __syncthreads();
    T* fl = fbuf + (size_t)buf * fsz + wl * FSP;   // this warp's line (padded)
    T* sl = sbuf + wl * FSP;
    const long long* lb = lbase + buf * TL;
    const bool valid = wl < TL && lb[wl] >= 0;
    auto F = [&](int k) -> T { return fl[k + k / R]; };

    if (wl < TL) {
      // ---- closures (FP64, lanes 0 and last) --------------------------------
      const int last = (n_rows - 1) / R;   // chunk holding the last row
      double bl0 = 0.0, bl1 = 0.0, br0 = 0.0, br1 = 0.0;
      if (!PERIODIC) {
        if (q == 0) {
          if (a.ovl) { bl0 = a.bcl0; bl1 = a.bcl1; }
          else {
            double fv[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) fv[k] = (double)F(k);
            bl0 = tb[16] * fv[0] + tb[17] * fv[1] + tb[18] * fv[2] + tb[19] * fv[3];
            bl1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
          }
        }
        if (q == last) {
          if (a.ovr) { br0 = a.bcr0; br1 = a.bcr1; }
          else {
            double fv[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) fv[k] = (double)F(n - 1 - k);
            br0 = tb[20] * fv[0] + tb[21] * fv[1] + tb[22] * fv[2] + tb[23] * fv[3];
            br1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
          }
        }
      }
      // ---- forward local sweep ------------------------------------------------
      V2<T> y[R];
      const int Nn = n - 1;
      const int off = PERIODIC ? 0 : 1;
      auto node = [&](int k) -> int {
        if (PERIODIC) { if (k < 0) return k + Nn; if (k >= Nn) return k - Nn; }
        return k;
      };
      V2<T> prev{T(0), T(0)};
      if (cnt > 0) {
        T fm = F(node(j0 + off - 1));
        T f0 = F(node(j0 + off));
#pragma unroll R
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (r < cnt) {
            const T fp = F(node(j + off + 1));
            V2<T> b{c1 * (fp - fm), c2 * ((fm - T(2) * f0) + fp)};
            if (!PERIODIC) {
              if (j == 0) {
                b.a = (T)((double)b.a - (tb[0] * bl0 + tb[1] * bl1));
                b.b = (T)((double)b.b - (tb[2] * bl0 + tb[3] * bl1));
              }
              if (j == n_rows - 1) {
                b.a = (T)((double)b.a - (tb[4] * br0 + tb[5] * br1));
                b.b = (T)((double)b.b - (tb[6] * br0 + tb[7] * br1));
              }
            }
            if (r == 0) {
              prev = b;
            } else if (in_head && j < H0) {
              const V2<T> q = mv(head + 20 * j, prev);
              prev = {b.a - q.a, b.b - q.b};
            } else {
              prev = {b.a - (Lf0 * prev.a + Lf1 * prev.b), b.b - (Lf2 * prev.a + Lf3 * prev.b)};
            }
            y[r] = prev;
            fm = f0;
            f0 = fp;
          }
        }
      }
      // ---- forward carry scan over lanes ---------------------------------------
      {
        Aff<T> m = aff_identity<T>();
        if (cnt > 0) {
          const int e = j0 + cnt;
          const T* Tm = (in_head && e - 1 < H0) ? head + 20 * (e - 1) + 12 : Phi + 4 * (cnt - 1);
          m = {Tm[0], Tm[1], Tm[2], Tm[3], prev.a, prev.b};
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const Aff<T> o = aff_shfl_up(m, d);
          if (lane >= d) m = aff_compose(m, o);
        }
        Aff<T> ex = aff_shfl_up(m, 1);
        if (lane == 0) ex = aff_identity<T>();
        T l0 = __shfl_sync(0xffffffffu, m.v0, 31), l1 = __shfl_sync(0xffffffffu, m.v1, 31);
        if (W > 1) {
          // the warps before this one: P = total_{wq-1} o ... o total_0
          if (lane == 31) s_tot[wl * W + wq] = m;
          __syncthreads();
          Aff<T> P = aff_identity<T>();
          for (int v = 0; v < wq; ++v) P = aff_compose(s_tot[wl * W + v], P);
          ex = aff_compose(ex, P);
          Aff<T> all = P;
          for (int v = wq; v < W; ++v) all = aff_compose(s_tot[wl * W + v], all);
          l0 = all.v0;
          l1 = all.v1;
          __syncthreads();   // s_tot is reused by the backward scan
        }
        V2<T> Yin{ex.v0, ex.v1};
        if (PERIODIC) {
          // ring closure: Y_{-1} = Gf * (scan result of the last chunk)
          const V2<T> ring = mv(Lfi + 16, V2<T>{l0, l1});
          Yin = {ex.v0 + ex.m0 * ring.a + ex.m1 * ring.b, ex.v1 + ex.m2 * ring.a + ex.m3 * ring.b};
        }
        if ((PERIODIC || q > 0) && cnt > 0) {
#pragma unroll R
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (r < cnt) {
              const T* mm = (in_head && j < H0) ? head + 20 * j + 12 : Phi + 4 * r;
              y[r].a += mm[0] * Yin.a + mm[1] * Yin.b;
              y[r].b += mm[2] * Yin.a + mm[3] * Yin.b;
            }
          }
        }
      }
      // ---- backward local sweep -----------------------------------------------
      V2<T> xn{T(0), T(0)};
#pragma unroll R
      for (int r = R - 1; r >= 0; --r) {
        const int j = j0 + r;
        if (r < cnt) {
          V2<T> x;
          if (in_head && j < H0) {
            const V2<T> pp = mv(head + 20 * j + 4, y[r]);
            const V2<T> qq = mv(head + 20 * j + 8, xn);
            x = {pp.a - qq.a, pp.b - qq.b};
          } else if (!PERIODIC && j == n_rows - 1) {
            x = mv(Plast, y[r]);
          } else {
            x = {(P0 * y[r].a + P1 * y[r].b) - (H0m * xn.a + H1m * xn.b),
                 (P2 * y[r].a + P3 * y[r].b) - (H2m * xn.a + H3m * xn.b)};
          }
          y[r] = x;
          xn = x;
        }
      }
      // ---- backward carry scan over lanes (suffix) -----------------------------------
      {
        Aff<T> m = aff_identity<T>();
        if (cnt > 0) {
          const T* Rm = (in_head && j0 < H0) ? head + 20 * j0 + 16 : Psi + 4 * cnt;
          m = {Rm[0], Rm[1], Rm[2], Rm[3], xn.a, xn.b};
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const Aff<T> o = aff_shfl_down(m, d);
          if (lane + d < 32) m = aff_compose(m, o);
        }
        Aff<T> ex = aff_shfl_down(m, 1);
        if (lane == 31) ex = aff_identity<T>();
        T l0 = __shfl_sync(0xffffffffu, m.v0, 0), l1 = __shfl_sync(0xffffffffu, m.v1, 0);
        if (W > 1) {
          // the warps after this one: Q = total_{wq+1} o ... o total_{W-1}
          if (lane == 0) s_tot[wl * W + wq] = m;
          __syncthreads();
          Aff<T> Q = aff_identity<T>();
          for (int v = W - 1; v > wq; --v) Q = aff_compose(s_tot[wl * W + v], Q);
          ex = aff_compose(ex, Q);
          Aff<T> all = Q;
          for (int v = wq; v >= 0; --v) all = aff_compose(s_tot[wl * W + v], all);
          l0 = all.v0;
          l1 = all.v1;
        }
        V2<T> Xin{ex.v0, ex.v1};
        if (PERIODIC) {
          const V2<T> ring = mv(Lfi + 20, V2<T>{l0, l1});
          Xin = {ex.v0 + ex.m0 * ring.a + ex.m1 * ring.b, ex.v1 + ex.m2 * ring.a + ex.m3 * ring.b};
        }
        if ((PERIODIC || q < last) && cnt > 0) {
#pragma unroll R
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (r < cnt) {
              const T* mm = (in_head && j < H0) ? head + 20 * j + 16 : Psi + 4 * (cnt - r);
              y[r].a += mm[0] * Xin.a + mm[1] * Xin.b;
              y[r].b += mm[2] * Xin.a + mm[3] * Xin.b;
            }
          }
        }
      }
      // ---- stage (d1, d2) in (own f line, sbuf line) --------------------------------------
      __syncwarp();
#pragma unroll R
      for (int r = 0; r < R; ++r) {
        if (r < cnt) {
          const int k = PERIODIC ? j0 + r : j0 + r + 1;
          fl[k + k / R] = y[r].a;
          sl[k + k / R] = y[r].b;
        }
      }
      if (!PERIODIC) {
        if (q == 0 && cnt > 0) {
          const double x0 = (double)y[0].a, x1 = (double)y[0].b;
          fl[0] = (T)((tb[8] * x0 + tb[9] * x1) + bl0);
          sl[0] = (T)((tb[10] * x0 + tb[11] * x1) + bl1);
        }
        if (q == last) {
#pragma unroll R
          for (int r = 0; r < R; ++r)
            if (r == cnt - 1) {
              const double x0 = (double)y[r].a, x1 = (double)y[r].b;
              const int k = n - 1;
              fl[k + k / R] = (T)((tb[12] * x0 + tb[13] * x1) + br0);
              sl[k + k / R] = (T)((tb[14] * x0 + tb[15] * x1) + br1);
            }
        }
      } else if (q == 0) {
        const int k = n - 1;
        fl[k + k / R] = y[0].a;
        sl[k + k / R] = y[0].b;
      }
      (void)valid;
    }
    __syncthreads();
    // ---- coalesced stores of the tile ---------------------------------------------------
    {
      const T* f1 = fbuf + (size_t)buf * fsz;
      auto metric = [&](int k, double& o1, double& o2) {
        if (J) {
          const double Jk = J[k], dJk = J[n + k];
          o2 = Jk * Jk * o2 + Jk * dJk * o1;
          o1 = Jk * o1;
        }
      };
      const int total = TL * n;
      if (CONTIG) {
        int l = threadIdx.x / n, k = threadIdx.x - (threadIdx.x / n) * n;
        const int step_l = blockDim.x / n, step_k = blockDim.x - step_l * n;
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
          const long long b = lb[l];
          if (b >= 0) {
            double o1 = (double)f1[l * FSP + k + k / R], o2 = (double)sbuf[l * FSP + k + k / R];
            metric(k, o1, o2);
            store_out<T>(a, b + k, o1, o2, k);
          }
          l += step_l;
          k += step_k;
          if (k >= n) { k -= n; ++l; }
        }
      } else {
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
          const int k = e >> a.tl_shift, l = e & (TL - 1);
          const long long b = lb[l];
          if (b >= 0) {
            double o1 = (double)f1[l * FSP + k + k / R], o2 = (double)sbuf[l * FSP + k + k / R];
            metric(k, o1, o2);
            store_out<T>(a, b + (int64_t)k * a.inner, o1, o2, k);
          }
        }
      }
    }
    __syncthreads();
    buf ^= (a.nbuf == 2) ? 1 : 0;
  }
  cp_async_wait<0>();
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

// ---- lane-per-line kernel ---------------------------------------------------------
//
// For many lines (3-D grids): lane l of a warp owns line 32g + l and runs the
// block-Thomas recurrences serially along it, so no scan, shuffle or carry
// fix-up is needed.  A line is cut into chunks of kLaneCR rows and visited
// twice:
//   pass 1: forward sweep y_r = b_r - Lf_r y_{r-1}; the carry at the end of
//           every chunk is kept in shared memory;
//   pass 2: chunks in reverse order: the forward sweep of the chunk is redone
//           from the stored carry (y in registers), then back substitution
//           x_r = P_r y_r - H_r x_{r+1} from the carry of the chunk after it.
// Each chunk's nodes (plus one halo node either side) are staged through a
// [rows][lanes] shared tile so global loads and stores are coalesced for the
// strided axes (lanes = adjacent lines) and the contiguous axis (lanes = nodes
// of one line).  Periodic axes close the forward recurrence exactly on the
// ring (Gf = (I - (-Lf)^N)^-1) and the backward one with the carry
// X = Gb x_0, where x_0 of the zero-carry sweep is the sum over the first
// kLaneK rows of (-H)^k P y_k (the neglected tail is below 0.46^64 of x_0).
constexpr int kLaneCR = 16;
constexpr int kLaneK = 64;

struct LaneTab {
  static constexpr int Lf = 0, P = 4, H = 8, Plast = 12, Gf = 16, Gb = 20, PhiC = 24, Q = 28, M = 32;
  static constexpr int head = M + 4 * kLaneK;   // per head row: Lf, P, H (12)
};

template <typename T>
__device__ __forceinline__ V2<T> mvs(const T* m, T a0, T a1) {
  return {m[0] * a0 + m[1] * a1, m[2] * a0 + m[3] * a1};
}

// The lane table holds the factors in a scaled form: with D = diag(a1/h, a2/h^2)
// the forward recurrence runs on y~ = D^-1 y, whose right-hand side is the
// plain differences (f+ - f-, f- - 2 f0 + f+); every factor that touches y is
// rescaled on the host (Lf~ = D^-1 Lf D, P~ = P D, ...), so no row pays for
// the RHS constants.
template <int N>
__device__ __forceinline__ void cp_async_wait_dyn(int pending) {
  // cp.async.wait_group takes an immediate: dispatch on the (small) count
  if (pending <= 0) cp_async_wait<0>();
  else if (pending == 1 || N <= 2) cp_async_wait<1>();
  else cp_async_wait<2>();
}

template <typename T, bool PERIODIC, bool PLAIN, int NBUF, bool CONTIG>
__global__ void __launch_bounds__(128) ccd_lane_kernel(CcdArgs a, const T* __restrict__ ltab_g, int ltab_total) {
  constexpr int CR = kLaneCR, TR = CR + 2;
  constexpr int TS = CONTIG ? 33 : 32;   // tile row stride (padded for the transposing copies)
  constexpr int NT = NBUF + (CONTIG ? 1 : 0);   // + the d2 output tile
  static_assert(NBUF == 2 || NBUF == 3, "f tile ring of 2 or 3 buffers");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* lt = reinterpret_cast<T*>(smem_raw);
  const int lt_pad = (ltab_total + 1) & ~1;
  const int n = a.n, n_rows = a.n_rows, H0 = PERIODIC ? 0 : a.H0;
  const int P = (n_rows + CR - 1) / CR;
  const int warps = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* fb0 = lt + lt_pad + (size_t)wid * (NT * TR * TS + 64 * P);   // ring of f tiles [TR][TS]
  T* dt = fb0 + NBUF * TR * TS;                                       // contiguous axis: d2 tile
  T* cy = fb0 + NT * TR * TS;                                         // chunk-end carries [P][2][32]
  stage_table<T>(lt, ltab_g, ltab_total);

  const T* __restrict__ f = static_cast<const T*>(a.f);
  const TabLayout lay{a.C, a.H0};
  const double* tb = a.tab + lay.bc();
  const double c1d = tb[30], c2d = tb[31];
  const T lf0 = lt[LaneTab::Lf], lf1 = lt[LaneTab::Lf + 1], lf2 = lt[LaneTab::Lf + 2], lf3 = lt[LaneTab::Lf + 3];
  const T p0 = lt[LaneTab::P], p1 = lt[LaneTab::P + 1], p2 = lt[LaneTab::P + 2], p3 = lt[LaneTab::P + 3];
  const T h0 = lt[LaneTab::H], h1 = lt[LaneTab::H + 1], h2 = lt[LaneTab::H + 2], h3 = lt[LaneTab::H + 3];
  const int Nn = n - 1;   // periodic: unique nodes
  const int64_t inner = a.inner;
  const int64_t n_groups = (a.n_lines + 31) / 32;
  const double* J = a.J;

  for (int64_t g = blockIdx.x * (int64_t)warps + wid; g < n_groups; g += (int64_t)gridDim.x * warps) {
    const int64_t L = g * 32 + lane;
    const bool act = L < a.n_lines;
    int64_t base = 0;
    if (act) {
      const int64_t o = L / inner, i = L - o * inner;
      base = o * (int64_t)n * inner + i;
    }
    const T* __restrict__ fl = f + base;
    // asynchronous copy of nodes k0 + t, t in [0, KN), into tile[t][lane]
    // FP64 strided axes: pass-1 chunks are staged with L2 evict_last (pass 2
    // re-reads them), pass-2 chunks and the reused last chunk with
    // evict_first (measured 2-3.5 % faster at 257^3; FP32 unchanged, so plain)
    const uint64_t pol_keep = pol_evict_last(), pol_last = pol_evict_first();
    auto stage = [&](T* tile, int k0, int KN, bool keep) {
      if (CONTIG) {
        // element e = (line ll, node t) of the chunk, e = lane + 32 i: runs of KN
        // contiguous nodes per line, so each warp copy reads ~2 contiguous runs
        int ll = lane / KN, t = lane - (lane / KN) * KN;
        const int dl = 32 / KN, dt_ = 32 - dl * KN;
        const T* fg = f + g * 32 * (int64_t)n;   // first line of the group
        const int nl = (a.n_lines - g * 32 < 32) ? (int)(a.n_lines - g * 32) : 32;
        const bool wrap = PERIODIC && (k0 < 0 || k0 + KN > Nn);
        for (int i = 0; i < KN; ++i) {
          if (ll < nl) {
            int kk = k0 + t;
            if (wrap) kk = (kk < 0) ? kk + Nn : (kk >= Nn ? kk - Nn : kk);
            cp_async<sizeof(T)>(tile + t * TS + ll, fg + (ll * n + kk), true);
          }
          ll += dl;
          t += dt_;
          if (t >= KN) { t -= KN; ++ll; }
        }
        cp_async_commit();
        return;
      }
      if (act) {
        if (PERIODIC && (k0 < 0 || k0 + KN > Nn)) {
          for (int t = 0; t < KN; ++t) {
            int k = k0 + t;
            k = (k < 0) ? k + Nn : (k >= Nn ? k - Nn : k);
            cp_async<sizeof(T)>(tile + t * TS + lane, fl + (int64_t)k * inner, true);
          }
        } else {
          const T* src = fl + (int64_t)k0 * inner;
          if (sizeof(T) == 8) {
            const uint64_t pol = keep ? pol_keep : pol_last;
            for (int t = 0; t < KN; ++t) {
              cp_async_pol<sizeof(T)>(tile + t * TS + lane, src, pol);
              src += inner;
            }
          } else {
            for (int t = 0; t < KN; ++t) {
              cp_async<sizeof(T)>(tile + t * TS + lane, src, true);
              src += inner;
            }
          }
        }
      }
      cp_async_commit();
    };
    auto put = [&](int k, double o1, double o2) {
      if (!act) return;
      if (J) {
        const double Jk = J[k], dJk = J[n + k];
        o2 = Jk * Jk * o2 + Jk * dJk * o1;
        o1 = Jk * o1;
      }
      store_out<T>(a, base + (int64_t)k * inner, o1, o2, k);
    };
    auto k0_of = [&](int c) { return PERIODIC ? c * CR - 1 : c * CR; };
    auto cnt_of = [&](int c) { return min(CR, n_rows - c * CR); };

    // chunk loads in visiting order: 0 .. P-1 (pass 1), then P-2 .. 0 (pass 2;
    // chunk P-1 is reused from pass 1); load l lives in ring buffer l % NBUF
    const int n_loads = 2 * P - 1;
    auto chunk_of_load = [&](int l) { return l < P ? l : 2 * P - 2 - l; };
    int issued = 0;
    // make load `need` resident, keeping up to NBUF - 1 loads ahead in flight
    auto acquire = [&](int need) -> const T* {
      const int want = min(n_loads, need + NBUF);
      while (issued < want) {
        const int c = chunk_of_load(issued);
        stage(fb0 + (issued % NBUF) * TR * TS, k0_of(c), cnt_of(c) + 2, issued < P - 1);
        ++issued;
      }
      cp_async_wait_dyn<NBUF>(issued - need - 1);
      __syncwarp();
      return fb0 + (need % NBUF) * TR * TS;
    };

    // wall closures (FP64): boundary pieces bl, br and their (scaled) RHS corrections
    double bl0 = 0.0, bl1 = 0.0, br0 = 0.0, br1 = 0.0;
    T cl0 = T(0), cl1 = T(0), cr0 = T(0), cr1 = T(0);
    if (!PERIODIC && act) {
      if (a.ovl) { bl0 = a.bcl0; bl1 = a.bcl1; }
      else {
        double fv[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) fv[k] = (double)fl[(int64_t)k * inner];
        bl0 = tb[16] * fv[0] + tb[17] * fv[1] + tb[18] * fv[2] + tb[19] * fv[3];
        bl1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
      }
      if (a.ovr) { br0 = a.bcr0; br1 = a.bcr1; }
      else {
        double fv[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) fv[k] = (double)fl[(int64_t)(n - 1 - k) * inner];
        br0 = tb[20] * fv[0] + tb[21] * fv[1] + tb[22] * fv[2] + tb[23] * fv[3];
        br1 = tb[24] * fv[0] + tb[25] * fv[1] + tb[26] * fv[2] + tb[27] * fv[3] + tb[28] * fv[4] + tb[29] * fv[5];
      }
      cl0 = (T)((tb[0] * bl0 + tb[1] * bl1) / c1d);
      cl1 = (T)((tb[2] * bl0 + tb[3] * bl1) / c2d);
      cr0 = (T)((tb[4] * br0 + tb[5] * br1) / c1d);
      cr1 = (T)((tb[6] * br0 + tb[7] * br1) / c2d);
    }
    // one forward row; SPECIAL rows carry closures / head factors / ring sums
    auto row_fwd = [&](int r, T fm, T f0, T fp, V2<T> yp, bool special) -> V2<T> {
      T ba = fp - fm, bb = (fm + fp) - T(2) * f0;
      if (special) {
        if (!PERIODIC) {
          if (r == 0) { ba -= cl0; bb -= cl1; }
          if (r == n_rows - 1) { ba -= cr0; bb -= cr1; }
          if (r < H0) {
            const T* m = lt + LaneTab::head + 12 * r;
            return {ba - (m[0] * yp.a + m[1] * yp.b), bb - (m[2] * yp.a + m[3] * yp.b)};
          }
        }
      }
      return {ba - (lf0 * yp.a + lf1 * yp.b), bb - (lf2 * yp.a + lf3 * yp.b)};
    };

    // ---- pass 1: forward sweep, chunk-end carries -------------------------------------
    V2<T> y{T(0), T(0)};
    V2<T> acc{T(0), T(0)};   // periodic: sum_{k < K} (-H)^k P~ y~_k of the zero-carry sweep
    for (int c = 0; c < P; ++c) {
      const T* tile = acquire(c);
      const int r0 = c * CR, cnt = cnt_of(c);
      T fm = tile[lane], f0 = tile[TS + lane];
      const bool special = cnt != CR || (PERIODIC ? (r0 < kLaneK) : (c == 0 || c == P - 1 || r0 < H0));
      if (!special) {
#pragma unroll
        for (int q = 0; q < CR; ++q) {
          const T fp = tile[(q + 2) * TS + lane];
          y = row_fwd(r0 + q, fm, f0, fp, y, false);
          fm = f0;
          f0 = fp;
        }
      } else {
        for (int q = 0; q < cnt; ++q) {
          const int r = r0 + q;
          const T fp = tile[(q + 2) * TS + lane];
          y = row_fwd(r, fm, f0, fp, y, true);
          if (PERIODIC && r < kLaneK) {
            const V2<T> u = mvs(lt + LaneTab::M + 4 * r, y.a, y.b);
            acc.a += u.a;
            acc.b += u.b;
          }
          fm = f0;
          f0 = fp;
        }
      }
      cy[(c * 2) * 32 + lane] = y.a;
      cy[(c * 2 + 1) * 32 + lane] = y.b;
      __syncwarp();
    }
    // ---- ring closures -------------------------------------------------------------
    V2<T> yin{T(0), T(0)}, xc{T(0), T(0)};
    if (PERIODIC) {
      yin = mvs(lt + LaneTab::Gf, y.a, y.b);
      V2<T> corr = yin;
      for (int c = 0; c + 1 < P; ++c) {
        corr = mvs(lt + LaneTab::PhiC, corr.a, corr.b);
        cy[(c * 2) * 32 + lane] += corr.a;
        cy[(c * 2 + 1) * 32 + lane] += corr.b;
      }
      const V2<T> qy = mvs(lt + LaneTab::Q, yin.a, yin.b);
      xc = mvs(lt + LaneTab::Gb, acc.a + qy.a, acc.b + qy.b);
      __syncwarp();
    }
    // ---- pass 2: chunks in reverse order ------------------------------------------------
    const int noff = PERIODIC ? 0 : 1;   // node of row r
    for (int c = P - 1; c >= 0; --c) {
      const T* tile = acquire(c == P - 1 ? P - 1 : 2 * P - 2 - c);
      const int r0 = c * CR, cnt = cnt_of(c);
      const bool special = !PERIODIC && (c == 0 || c == P - 1 || r0 < H0);
      V2<T> yr[CR];
      V2<T> xlast{T(0), T(0)};
      V2<T> yp = (c == 0) ? yin : V2<T>{cy[((c - 1) * 2) * 32 + lane], cy[((c - 1) * 2 + 1) * 32 + lane]};
      T fm = tile[lane], f0 = tile[TS + lane];
      if (!special && cnt == CR) {
#pragma unroll
        for (int q = 0; q < CR; ++q) {
          const T fp = tile[(q + 2) * TS + lane];
          yp = row_fwd(r0 + q, fm, f0, fp, yp, false);
          yr[q] = yp;
          fm = f0;
          f0 = fp;
        }
        __syncwarp();   // the tile is refilled by the prefetch after next
#pragma unroll
        for (int q = CR - 1; q >= 0; --q) {
          const V2<T> x{(p0 * yr[q].a + p1 * yr[q].b) - (h0 * xc.a + h1 * xc.b),
                        (p2 * yr[q].a + p3 * yr[q].b) - (h2 * xc.a + h3 * xc.b)};
          xc = x;
          yr[q] = x;
        }
      } else {
#pragma unroll
        for (int q = 0; q < CR; ++q) {
          if (q < cnt) {
            const T fp = tile[(q + 2) * TS + lane];
            yp = row_fwd(r0 + q, fm, f0, fp, yp, true);
            yr[q] = yp;
            fm = f0;
            f0 = fp;
          }
        }
        __syncwarp();
#pragma unroll
        for (int q = CR - 1; q >= 0; --q) {
          if (q < cnt) {
            const int r = r0 + q;
            V2<T> x;
            if (!PERIODIC && r == n_rows - 1) {
              x = mvs(lt + LaneTab::Plast, yr[q].a, yr[q].b);
              xlast = x;
            } else if (r < H0) {
              const T* pm = lt + LaneTab::head + 12 * r + 4;
              const T* hm = pm + 4;
              x = {(pm[0] * yr[q].a + pm[1] * yr[q].b) - (hm[0] * xc.a + hm[1] * xc.b),
                   (pm[2] * yr[q].a + pm[3] * yr[q].b) - (hm[2] * xc.a + hm[3] * xc.b)};
            } else {
              x = {(p0 * yr[q].a + p1 * yr[q].b) - (h0 * xc.a + h1 * xc.b),
                   (p2 * yr[q].a + p3 * yr[q].b) - (h2 * xc.a + h3 * xc.b)};
            }
            xc = x;
            yr[q] = x;
          }
        }
      }
      if (CONTIG) {
        // results through the (consumed) f tile and the d2 tile, then runs of
        // contiguous nodes per line
        T* ot = const_cast<T*>(tile);
#pragma unroll
        for (int q = 0; q < CR; ++q) {
          if (q < cnt) {
            ot[(q + 1) * TS + lane] = yr[q].a;
            dt[(q + 1) * TS + lane] = yr[q].b;
          }
        }
        int t0 = 1, t1 = cnt + 1;
        if (!PERIODIC && c == P - 1) {
          const double x0 = (double)xlast.a, x1 = (double)xlast.b;
          ot[(cnt + 1) * TS + lane] = (T)((tb[12] * x0 + tb[13] * x1) + br0);
          dt[(cnt + 1) * TS + lane] = (T)((tb[14] * x0 + tb[15] * x1) + br1);
          t1 = cnt + 2;
        }
        if (!PERIODIC && c == 0) {
          const double x0 = (double)xc.a, x1 = (double)xc.b;
          ot[lane] = (T)((tb[8] * x0 + tb[9] * x1) + bl0);
          dt[lane] = (T)((tb[10] * x0 + tb[11] * x1) + bl1);
          t0 = 0;
        }
        __syncwarp();
        const int KN = t1 - t0;
        const int k0 = k0_of(c) + t0;
        int ll = lane / KN, t = lane - (lane / KN) * KN;
        const int dl = 32 / KN, dt_ = 32 - dl * KN;
        const int64_t g0 = g * 32 * (int64_t)n;
        const int nl = (a.n_lines - g * 32 < 32) ? (int)(a.n_lines - g * 32) : 32;
        const bool plain_c = a.d1 && a.d2 && !a.vd_out && !J;
        T* o1p = static_cast<T*>(a.d1) + g0;
        T* o2p = static_cast<T*>(a.d2) + g0;
        if (a.cr_out) {
          // corrector epilogue: all of this run's u* and rho first, then the
          // stores (see the strided branch)
          double pu[CR + 2], pr[CR + 2];
          int l2 = ll, t2 = t;
#pragma unroll
          for (int i = 0; i < CR + 2; ++i) {
            pu[i] = 0.0;
            pr[i] = 1.0;
            if (i < KN && l2 < nl) {
              const int64_t gi = g0 + (int64_t)l2 * n + k0 + t2;
              pu[i] = (double)static_cast<const T*>(a.cr_u)[gi];
              pr[i] = (double)static_cast<const T*>(a.cr_rho)[gi];
            }
            l2 += dl;
            t2 += dt_;
            if (t2 >= KN) { t2 -= KN; ++l2; }
          }
#pragma unroll
          for (int i = 0; i < CR + 2; ++i) {
            if (i < KN && ll < nl) {
              const int node = k0 + t;
              double o1 = (double)ot[(t0 + t) * TS + ll];
              if (J) o1 = J[node] * o1;
              double v = pu[i];
              if (!(a.cr_wall && (node == 0 || node == n - 1))) v = __dsub_rn(pu[i], __dmul_rn(a.cr_dt / pr[i], o1));
              static_cast<T*>(a.cr_out)[g0 + (int64_t)ll * n + node] = (T)v;
            }
            ll += dl;
            t += dt_;
            if (t >= KN) { t -= KN; ++ll; }
          }
        } else if (a.vd_out) {
          // variable-density epilogue: operands first, then the stores
          double pr[CR + 2], pdr[CR + 2], po[CR + 2];
          int l2 = ll, t2 = t;
#pragma unroll
          for (int i = 0; i < CR + 2; ++i) {
            pr[i] = 1.0;
            pdr[i] = 0.0;
            po[i] = 0.0;
            if (i < KN && l2 < nl) {
              const int64_t gi = g0 + (int64_t)l2 * n + k0 + t2;
              pr[i] = (double)static_cast<const T*>(a.vd_rho)[gi];
              pdr[i] = (double)static_cast<const T*>(a.vd_drho)[gi];
              if (a.vd_accumulate) po[i] = (double)static_cast<const T*>(a.vd_out)[gi];
            }
            l2 += dl;
            t2 += dt_;
            if (t2 >= KN) { t2 -= KN; ++l2; }
          }
#pragma unroll
          for (int i = 0; i < CR + 2; ++i) {
            if (i < KN && ll < nl) {
              const int node = k0 + t;
              double o1 = (double)ot[(t0 + t) * TS + ll], o2 = (double)dt[(t0 + t) * TS + ll];
              if (J) {
                const double Jk = J[node], dJk = J[n + node];
                o2 = Jk * Jk * o2 + Jk * dJk * o1;
                o1 = Jk * o1;
              }
              const double r = pr[i];
              double tv = o2 / r - (pdr[i] / (r * r)) * o1;
              if (a.vd_accumulate) tv = po[i] + tv;
              static_cast<T*>(a.vd_out)[g0 + (int64_t)ll * n + node] = (T)tv;
            }
            ll += dl;
            t += dt_;
            if (t >= KN) { t -= KN; ++ll; }
          }
        } else
        for (int i = 0; i < KN; ++i) {
          if (ll < nl) {
            const int node = k0 + t;
            const T v1 = ot[(t0 + t) * TS + ll], v2 = dt[(t0 + t) * TS + ll];
            if (plain_c) {
              o1p[ll * n + node] = v1;
              o2p[ll * n + node] = v2;
            } else {
              double o1 = (double)v1, o2 = (double)v2;
              if (J) {
                const double Jk = J[node], dJk = J[n + node];
                o2 = Jk * Jk * o2 + Jk * dJk * o1;
                o1 = Jk * o1;
              }
              store_out<T>(a, g0 + (int64_t)ll * n + node, o1, o2, node);
            }
          }
          ll += dl;
          t += dt_;
          if (t >= KN) { t -= KN; ++ll; }
        }
        if (PERIODIC && c == 0) put(Nn, (double)xc.a, (double)xc.b);   // image node N = node 0 (own line)
        __syncwarp();
        continue;
      }
      // ascending burst of coalesced stores (lanes = adjacent lines)
      if (PLAIN) {
        if (act) {
          T* o1 = static_cast<T*>(a.d1) + base + (int64_t)(r0 + noff) * inner;
          T* o2 = static_cast<T*>(a.d2) + base + (int64_t)(r0 + noff) * inner;
#pragma unroll
          for (int q = 0; q < CR; ++q) {
            if (q < cnt) {
              __stcs(o1, yr[q].a);   // streaming: keep L2 for the lines pass 2 re-reads
              __stcs(o2, yr[q].b);
              o1 += inner;
              o2 += inner;
            }
          }
        }
      } else if (a.cr_out) {
        // corrector epilogue: the chunk's u* and rho are loaded before any
        // store (the stores may alias u*, which would otherwise serialize each
        // node's loads behind the previous node's store)
        if (act) {
          const int64_t o0 = base + (int64_t)(r0 + noff) * inner;
          const T* cu = static_cast<const T*>(a.cr_u) + o0;
          const T* crh = static_cast<const T*>(a.cr_rho) + o0;
          T* co = static_cast<T*>(a.cr_out) + o0;
          double pu[CR], pr[CR];
#pragma unroll
          for (int q = 0; q < CR; ++q) {
            pu[q] = 0.0;
            pr[q] = 1.0;
            if (q < cnt) {
              pu[q] = (double)cu[(int64_t)q * inner];
              pr[q] = (double)crh[(int64_t)q * inner];
            }
          }
#pragma unroll
          for (int q = 0; q < CR; ++q) {
            if (q < cnt) {
              const int k = r0 + q + noff;
              double o1 = (double)yr[q].a;
              if (J) o1 = J[k] * o1;
              double v = pu[q];
              if (!(a.cr_wall && (k == 0 || k == n - 1))) v = __dsub_rn(pu[q], __dmul_rn(a.cr_dt / pr[q], o1));
              co[(int64_t)q * inner] = (T)v;
            }
          }
        }
      } else if (a.vd_out) {
        // variable-density epilogue: operands first, then the stores (as above)
        if (act) {
          const int64_t o0 = base + (int64_t)(r0 + noff) * inner;
          const T* vr = static_cast<const T*>(a.vd_rho) + o0;
          const T* vdr = static_cast<const T*>(a.vd_drho) + o0;
          T* vo = static_cast<T*>(a.vd_out) + o0;
          double pr[CR], pdr[CR], po[CR];
#pragma unroll
          for (int q = 0; q < CR; ++q) {
            pr[q] = 1.0;
            pdr[q] = 0.0;
            po[q] = 0.0;
            if (q < cnt) {
              pr[q] = (double)vr[(int64_t)q * inner];
              pdr[q] = (double)vdr[(int64_t)q * inner];
              if (a.vd_accumulate) po[q] = (double)vo[(int64_t)q * inner];
            }
          }
#pragma unroll
          for (int q = 0; q < CR; ++q) {
            if (q < cnt) {
              const int k = r0 + q + noff;
              double o1 = (double)yr[q].a, o2 = (double)yr[q].b;
              if (J) {
                const double Jk = J[k], dJk = J[n + k];
                o2 = Jk * Jk * o2 + Jk * dJk * o1;
                o1 = Jk * o1;
              }
              const double r = pr[q];
              double tv = o2 / r - (pdr[q] / (r * r)) * o1;
              if (a.vd_accumulate) tv = po[q] + tv;
              vo[(int64_t)q * inner] = (T)tv;
            }
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < CR; ++q)
          if (q < cnt) put(r0 + q + noff, (double)yr[q].a, (double)yr[q].b);
      }
      if (!PERIODIC && c == P - 1) {
        const double x0 = (double)xlast.a, x1 = (double)xlast.b;
        put(n - 1, (tb[12] * x0 + tb[13] * x1) + br0, (tb[14] * x0 + tb[15] * x1) + br1);
      }
      if (c == 0) {
        if (!PERIODIC) {
          const double x0 = (double)xc.a, x1 = (double)xc.b;
          put(0, (tb[8] * x0 + tb[9] * x1) + bl0, (tb[10] * x0 + tb[11] * x1) + bl1);
        } else {
          put(Nn, (double)xc.a, (double)xc.b);   // image node N = node 0
        }
      }
      __syncwarp();   // this tile may be refilled by the next acquire
    }
    cp_async_wait<0>();
    __syncwarp();
  }
}

int build_tables(tpf_ccd_plan* p, std::vector<double>& tab) {
  const double h = p->h;
  const int n_rows = p->n_rows;
  const int C = p->C;
  const M2 L = {kAlpha1, kB1 * h, kB2 / h, kBeta2};
  const M2 U = {kAlpha1, -kB1 * h, -kB2 / h, kBeta2};
  const M2 Ml = {-1.5, 1.5 * h, 0.0, 0.0};
  const M2 Mr = {-1.5, -1.5 * h, 0.0, 0.0};
  // fixed point of LU = I - L LU^-1 U (interior block-LU factor)
  M2 LUi = eye();
  for (int it = 0; it < 400; ++it) LUi = sub(eye(), mul(mul(L, inv(LUi)), U));
  const M2 Pinf = inv(LUi), Lfinf = mul(L, Pinf), Hinf = mul(Pinf, U);
  const int P = (n_rows + C - 1) / C;
  int H0 = 0;
  std::vector<M2> Lf, Pm, Hm;
  if (p->bc == TPF_BC_WALL) {
    // per-row factors of the folded system (ccd_solver_helpers.py:238-245)
    std::vector<M2> LU(n_rows);
    Lf.resize(n_rows); Pm.resize(n_rows); Hm.resize(n_rows);
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
      const double dt = det(LU[j]);
      if (!std::isfinite(dt) || std::fabs(dt) < 1e-300) {
        tpf::set_error("CCD block-tridiagonal factorization encountered a singular pivot at block %d", j);
        return TPF_ESINGULAR;
      }
      Pm[j] = inv(LU[j]);
      Hm[j] = (j < n_rows - 1) ? mul(Pm[j], U) : M2{0, 0, 0, 0};
    }
    // smallest head (a multiple of C) beyond which the factors sit at the fixed point
    H0 = n_rows;
    for (int hh = C; hh < n_rows; hh += C) {
      // rows >= hh use the fixed-point Lf (all rows, the last included) and
      // the fixed-point P, H (all but the last, which carries the closure)
      bool conv = true;
      for (int j = hh; j < n_rows && conv; ++j) {
        double e = maxabs(sub(Lf[j], Lfinf)) / maxabs(Lfinf);
        if (j < n_rows - 1)
          e = std::max(e, std::max(maxabs(sub(Pm[j], Pinf)) / maxabs(Pinf), maxabs(sub(Hm[j], Hinf)) / maxabs(Hinf)));
        conv = e < 1e-15;
      }
      if (conv) { H0 = hh; break; }
    }
  }
  TabLayout lay{C, H0};
  tab.assign(lay.total(), 0.0);
  // Phi_k = (-Lf)^(k+1), Psi_k = (-H)^k in the fixed-point region
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
  if (p->bc == TPF_BC_WALL) {
    for (int q = 0; q < 4; ++q) tab[lay.cst() + 12 + q] = Pm[n_rows - 1][q];
    // head rows: Lf, P, H and the chunk-relative transfer products
    //   PhiH_j = prod_{m=s..j} (-Lf_m),  PsiH_j = prod_{m=j..e-1} (-H_m)
    for (int cc = 0; cc * C < H0; ++cc) {
      const int s = cc * C, e = std::min(s + C, n_rows);
      M2 ph = eye();
      for (int j = s; j < e; ++j) {
        ph = mul(neg(Lf[j]), ph);
        for (int q = 0; q < 4; ++q) tab[lay.head() + 20 * j + 12 + q] = ph[q];
      }
      M2 ps = eye();
      for (int j = e - 1; j >= s; --j) {
        ps = mul(neg(Hm[j]), ps);
        for (int q = 0; q < 4; ++q) tab[lay.head() + 20 * j + 16 + q] = ps[q];
      }
      for (int j = s; j < e; ++j)
        for (int q = 0; q < 4; ++q) {
          tab[lay.head() + 20 * j + q] = Lf[j][q];
          tab[lay.head() + 20 * j + 4 + q] = Pm[j][q];
          tab[lay.head() + 20 * j + 8 + q] = Hm[j][q];
        }
    }
  } else {
    // ring transfers of the two cyclic recurrences
    M2 Tr = eye(), Rr = eye();
    for (int cc = 0; cc < P; ++cc) {
      const int s = cc * C, e = std::min(s + C, n_rows);
      M2 Tc, Rc;
      for (int q = 0; q < 4; ++q) {
        Tc[q] = tab[lay.phi() + 4 * (e - s - 1) + q];
        Rc[q] = tab[lay.psi() + 4 * (e - s) + q];
      }
      Tr = mul(Tc, Tr);   // T_{P-1} ... T_0
      Rr = mul(Rr, Rc);   // R_0 R_1 ... R_{P-1}
    }
    const M2 Gf = inv(sub(eye(), Tr)), Gb = inv(sub(eye(), Rr));
    for (int q = 0; q < 4; ++q) {
      tab[lay.cst() + 16 + q] = Gf[q];
      tab[lay.cst() + 20 + q] = Gb[q];
    }
  }
  // closure constants (ccd_solver.py:408-456)
  const int b = lay.bc();
  for (int q = 0; q < 4; ++q) {
    tab[b + q] = L[q];
    tab[b + 4 + q] = U[q];
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
  p->P = P;
  p->H0 = H0;
  // lane-per-line kernel table, scaled by D = diag(a1/h, a2/h^2) (see ccd_lane_kernel)
  {
    const double d[2] = {kA1 / h, kA2 / (h * h)};
    auto sim = [&](const M2& m) {   // D^-1 m D
      return M2{m[0], m[1] * d[1] / d[0], m[2] * d[0] / d[1], m[3]};
    };
    auto rmul = [&](const M2& m) {  // m D
      return M2{m[0] * d[0], m[1] * d[1], m[2] * d[0], m[3] * d[1]};
    };
    const int tot = LaneTab::head + 12 * H0;
    std::vector<double>& lt = p->ltab_host;
    lt.assign(tot, 0.0);
    const M2 Lfs = sim(Lfinf), Ps = rmul(Pinf);
    for (int q = 0; q < 4; ++q) {
      lt[LaneTab::Lf + q] = Lfs[q];
      lt[LaneTab::P + q] = Ps[q];
      lt[LaneTab::H + q] = Hinf[q];
    }
    if (p->bc == TPF_BC_WALL) {
      const M2 Pl = rmul(Pm[n_rows - 1]);
      for (int q = 0; q < 4; ++q) lt[LaneTab::Plast + q] = Pl[q];
      for (int j = 0; j < H0; ++j) {
        const M2 lj = sim(Lf[j]), pj = rmul(Pm[j]);
        for (int q = 0; q < 4; ++q) {
          lt[LaneTab::head + 12 * j + q] = lj[q];
          lt[LaneTab::head + 12 * j + 4 + q] = pj[q];
          lt[LaneTab::head + 12 * j + 8 + q] = Hm[j][q];
        }
      }
    } else {
      // ring: Tr = (-Lf)^N, Rr = (-H)^N; PhiC = (-Lf)^CR; M_k = (-H)^k P; Q = sum_k M_k (-Lf)^(k+1)
      M2 Tr = eye(), Rr = eye(), PhiC = eye();
      for (int k = 0; k < n_rows; ++k) {
        Tr = mul(neg(Lfinf), Tr);
        Rr = mul(neg(Hinf), Rr);
      }
      for (int k = 0; k < kLaneCR; ++k) PhiC = mul(neg(Lfinf), PhiC);
      const M2 Gf = inv(sub(eye(), Tr)), Gb = inv(sub(eye(), Rr));
      M2 Hk = eye(), Phk = eye(), Q = {0, 0, 0, 0};
      const int K = std::min(kLaneK, n_rows);
      for (int k = 0; k < K; ++k) {
        const M2 Mk = mul(Hk, Pinf);
        Phk = mul(neg(Lfinf), Phk);
        Q = add(Q, mul(Mk, Phk));
        const M2 Mks = rmul(Mk);
        for (int q = 0; q < 4; ++q) lt[LaneTab::M + 4 * k + q] = Mks[q];
        Hk = mul(neg(Hinf), Hk);
      }
      const M2 Gfs = sim(Gf), PhiCs = sim(PhiC), Qs = rmul(Q);
      for (int q = 0; q < 4; ++q) {
        lt[LaneTab::Gf + q] = Gfs[q];
        lt[LaneTab::Gb + q] = Gb[q];
        lt[LaneTab::PhiC + q] = PhiCs[q];
        lt[LaneTab::Q + q] = Qs[q];
      }
    }
  }
  return TPF_OK;
}

struct LaunchShape {
  int TL, LS, FS, nbuf, grid;
  size_t smem;
};

template <typename T>
size_t smem_bytes(const tpf_ccd_plan* p, bool contig, int TL, int nbuf, int LS, int FS) {
  TabLayout lay{p->C, p->H0};
  const size_t fsz = contig ? (size_t)TL * FS : (size_t)TL * p->n_pts;
  return sizeof(double) * 4 * TL + sizeof(long long) * 2 * TL +
         sizeof(T) * (((size_t)lay.total() + 1) & ~(size_t)1) + sizeof(T) * (((size_t)TL * LS + 1) & ~(size_t)1) +
         sizeof(T) * nbuf * fsz + sizeof(T) * (size_t)p->P * TL * 4 + 64;
}

template <typename T>
LaunchShape pick_shape(const tpf_ccd_plan* p, bool contig, int64_t n_lines) {
  const int n = (int)p->n_pts;
  const int LS = 2 * p->n_rows + 1;
  const int FS = (n % 2) ? n : n + 1;
  const int nsm = tpf::sm_count();
  LaunchShape best{};
  best.TL = 0;
  double best_score = -1e30;
  const int tl_opts[6] = {32, 16, 8, 4, 2, 1};
  for (int t = 0; t < 6; ++t) {
    const int TL = tl_opts[t];
    if (TL * p->P > 512) continue;
    const int64_t tiles = (n_lines + TL - 1) / TL;
    for (int nbuf = 2; nbuf >= 1; --nbuf) {
      const size_t sm = smem_bytes<T>(p, contig, TL, nbuf, LS, FS);
      if (sm > 225 * 1024) continue;
      const int per_sm = std::max(1, (int)std::min<size_t>(8, (228 * 1024) / (sm + 1024)));
      const int64_t slots = (int64_t)nsm * per_sm;
      const int64_t grid = std::min<int64_t>(tiles, slots);
      // score: enough resident threads, full waves, prefetch when CTAs own >1 tile
      const double waves = (double)tiles / (double)grid;
      const double threads_per_sm = (double)std::min<int64_t>(per_sm, (grid + nsm - 1) / nsm) * TL * p->P;
      double score = std::min(threads_per_sm, 512.0) + (nbuf == 2 && waves > 1.5 ? 200.0 : 0.0) +
                     (grid >= nsm ? 100.0 : 100.0 * grid / nsm);
      if (nbuf == 2 && waves <= 1.0) score -= 300.0;   // a second buffer without a second tile is waste
      if (score > best_score) {
        best_score = score;
        best = {TL, LS, FS, nbuf, (int)grid, sm};
      }
    }
  }
  return best;
}

template <typename T, int R>
LaunchShape pick_warp_shape(const tpf_ccd_plan* p, int64_t n_lines, int W) {
  const int n = (int)p->n_pts;
  int FSP = n + (n - 1) / R + 1;
  if (FSP % 2 == 0) ++FSP;
  const int nsm = tpf::sm_count();
  const int regs = R == 8 ? 128 : (R == 16 ? 168 : 255);
  TabLayout lay{R, p->H0};
  LaunchShape best{};
  best.TL = 0;
  double best_score = -1e30;
  const int tl_opts[4] = {8, 4, 2, 1};
  for (int t = 0; t < 4; ++t) {
    const int TL = tl_opts[t];
    const int threads = 32 * W * TL;
    if (threads > 256) continue;
    const int64_t tiles = (n_lines + TL - 1) / TL;
    const size_t fsz = (size_t)TL * FSP;
    for (int nbuf = 2; nbuf >= 1; --nbuf) {
      const size_t sm = sizeof(long long) * 2 * TL + sizeof(T) * (((size_t)lay.total() + 1) & ~(size_t)1) +
                        sizeof(T) * (nbuf + 1) * fsz + 64;
      if (sm > 225 * 1024) continue;
      const int by_smem = (int)((228 * 1024) / (sm + 1024));
      const int by_regs = 65536 / (regs * threads);
      const int per_sm = std::max(1, std::min(std::min(by_smem, by_regs), 16));
      const int64_t grid = std::min<int64_t>(tiles, (int64_t)nsm * per_sm);
      const double waves = (double)tiles / (double)grid;
      double score = 400.0 * std::min(1.0, (double)grid / nsm) + 0.25 * std::min(per_sm * threads, 2048) +
                     (nbuf == 2 && waves > 1.5 ? 150.0 : 0.0) - (nbuf == 2 && waves <= 1.0 ? 300.0 : 0.0);
      if (score > best_score) {
        best_score = score;
        best = {TL, 0, FSP, nbuf, (int)grid, sm};
      }
    }
  }
  return best;
}

// launch shape of the warp kernel for one (lines per block, tile buffers) choice
template <typename T, int R>
LaunchShape warp_shape(const tpf_ccd_plan* p, int64_t n_lines, int W, int TL, int nbuf) {
  const int n = (int)p->n_pts;
  int FSP = n + (n - 1) / R + 1;
  if (FSP % 2 == 0) ++FSP;
  const int nsm = tpf::sm_count();
  const int regs = R == 8 ? 128 : (R == 16 ? 168 : 255);
  TabLayout lay{R, p->H0};
  LaunchShape out{};
  out.TL = 0;
  const int threads = 32 * W * TL;
  if (threads > 256) return out;
  const size_t fsz = (size_t)TL * FSP;
  const size_t sm = sizeof(long long) * 2 * TL + sizeof(T) * (((size_t)lay.total() + 1) & ~(size_t)1) +
                    sizeof(T) * (nbuf + 1) * fsz + 64;
  if (sm > 225 * 1024) return out;
  const int by_smem = (int)((228 * 1024) / (sm + 1024));
  const int by_regs = 65536 / (regs * threads);
  const int per_sm = std::max(1, std::min(std::min(by_smem, by_regs), 16));
  const int64_t tiles = (n_lines + TL - 1) / TL;
  const int64_t grid = std::min<int64_t>(tiles, (int64_t)nsm * per_sm);
  out = {TL, 0, FSP, nbuf, (int)grid, sm};
  return out;
}

// many lines (3-D grids) and long enough lines: the lane-per-line kernel
bool use_lane_kernel(const tpf_ccd_plan* p, int64_t n_lines, bool periodic, bool contig) {
  if (p->n_rows < 128 || p->n_rows > 2048) return false;
  if (periodic != (p->bc == TPF_BC_PERIODIC)) return false;   // closure overrides on a periodic plan
  return n_lines >= 148LL * 4 * 32;
}

// Launch shape of the lane kernel: warps per block, f-tile ring depth, cap on
// resident blocks per SM.  Every shape computes each line with the same
// arithmetic, so the results are bitwise identical; only the speed differs.
using LaneShape = LaneShape_;

template <typename T>
using LaneFn = void (*)(CcdArgs, const T*, int);

template <typename T, int NB>
LaneFn<T> lane_fn_nb(bool periodic, bool plain, bool contig) {
  if (contig)
    return periodic ? ccd_lane_kernel<T, true, false, NB, true> : ccd_lane_kernel<T, false, false, NB, true>;
  if (periodic) return plain ? ccd_lane_kernel<T, true, true, NB, false> : ccd_lane_kernel<T, true, false, NB, false>;
  return plain ? ccd_lane_kernel<T, false, true, NB, false> : ccd_lane_kernel<T, false, false, NB, false>;
}

template <typename T>
int run_lane(const tpf_ccd_plan* p, const CcdArgs& a, bool periodic, bool contig, const LaneShape& sh,
             cudaStream_t stream) {
  const int W = sh.warps;
  const int P = (p->n_rows + kLaneCR - 1) / kLaneCR;
  const size_t per_warp = (size_t)(sh.nbuf + (contig ? 1 : 0)) * (kLaneCR + 2) * (contig ? 33 : 32) + 64 * (size_t)P;
  const size_t smem = sizeof(T) * ((((size_t)p->ltab_total + 1) & ~(size_t)1) + W * per_warp);
  TPF_CHECK_ARG(smem <= 225 * 1024, "CCD lane kernel: axis of %lld points needs too much shared memory",
                (long long)p->n_pts);
  const bool plain = a.d1 && a.d2 && !a.vd_out && !a.J;
  LaneFn<T> kern = sh.nbuf == 2 ? lane_fn_nb<T, 2>(periodic, plain, contig) : lane_fn_nb<T, 3>(periodic, plain, contig);
  TPF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  TPF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * W, smem));
  per_sm = std::max(1, std::min(per_sm, sh.max_bps));
  const int64_t groups = (a.n_lines + 31) / 32;
  const int64_t blocks = std::min<int64_t>((groups + W - 1) / W, (int64_t)tpf::sm_count() * per_sm);
  const T* lt = std::is_same<T, double>::value ? reinterpret_cast<const T*>(p->d_ltab)
                                               : reinterpret_cast<const T*>(p->d_ltabf);
  kern<<<(unsigned)blocks, 32 * W, smem, stream>>>(a, lt, p->ltab_total);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// Autotuner: on the first call of a (lines, axis kind, boundary, epilogue,
// dtype) combination, time the candidate shapes with CUDA events (one warm-up
// and two timed launches each) and keep the fastest in the plan.  Skipped while
// the stream is being captured into a graph (the default shape runs).
template <typename T>
int launch_lane(const tpf_ccd_plan* p, const CcdArgs& a, bool periodic, bool contig, cudaStream_t stream) {
  const bool plain = a.d1 && a.d2 && !a.vd_out && !a.J;
  const uint64_t key = ((uint64_t)a.n_lines << 8) | ((uint64_t)contig << 0) | ((uint64_t)periodic << 1) |
                       ((uint64_t)plain << 2) | ((uint64_t)(sizeof(T) == 8) << 3);
  auto it = p->lane_tuned.find(key);
  if (it != p->lane_tuned.end()) return run_lane<T>(p, a, periodic, contig, it->second, stream);
  const LaneShape def{4, std::is_same<T, double>::value ? 3 : 2, 64};
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  TPF_CUDA_TRY(cudaStreamIsCapturing(stream, &cs));
  // an accumulating (or in-place) epilogue must run exactly once: no tuning runs for it
  if (!p->autotune || cs != cudaStreamCaptureStatusNone || (a.vd_out && a.vd_accumulate) ||
      (a.cr_out && a.cr_out == a.cr_u))
    return run_lane<T>(p, a, periodic, contig, def, stream);
  const LaneShape cand[] = {{4, 3, 64}, {4, 2, 64}, {4, 3, 2}, {4, 2, 3}, {2, 3, 64}, {2, 2, 64}, {4, 2, 2}};
  cudaEvent_t e0, e1;
  TPF_CUDA_TRY(cudaEventCreate(&e0));
  TPF_CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  LaneShape bs = def;
  int st = TPF_OK;
  for (const LaneShape& c : cand) {
    if ((st = run_lane<T>(p, a, periodic, contig, c, stream))) {
      if (st != TPF_EINVAL) break;
      st = TPF_OK;   // a shape that does not fit in shared memory is skipped
      continue;
    }
    cudaEventRecord(e0, stream);
    for (int r = 0; r < 2 && !st; ++r) st = run_lane<T>(p, a, periodic, contig, c, stream);
    cudaEventRecord(e1, stream);
    if (cudaEventSynchronize(e1) != cudaSuccess || st) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      bs = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  p->lane_tuned[key] = bs;
  // the results of the last candidate are already in place and identical for every shape
  return TPF_OK;
}

template <typename T>
int launch_ccd(const tpf_ccd_plan* p, int64_t outer, int64_t inner, const void* f, void* d1, void* d2,
               const double* bcl, const double* bcr, int flags, cudaStream_t stream,
               const void* vd_rho = nullptr, const void* vd_drho = nullptr, void* vd_out = nullptr,
               int vd_accumulate = 0, const CcdArgs* corrector = nullptr) {
  const bool contig = (inner == 1);
  const int64_t n_lines = outer * inner;
  if (n_lines == 0) return TPF_OK;
  TPF_CHECK_ARG(f != d1 && f != d2 && f != vd_out, "the CCD input must not alias an output array");
  TPF_CHECK_ARG(!corrector || (f != corrector->cr_out && f != corrector->cr_u && f != corrector->cr_rho),
                "the pressure must not alias the velocity or density arrays");
  TPF_CHECK_ARG(n_lines < ((int64_t)1 << 31), "too many lines");
  // warp kernel: chunks of 8 rows, 1, 2 or 4 warps per line (lines up to 1024 rows)
  const bool warp = p->C == 8 && p->n_rows <= 32 * 8 * 4;
  const int W = p->n_rows <= 256 ? 1 : (p->n_rows <= 512 ? 2 : 4);
  LaunchShape s = !warp ? pick_shape<T>(p, contig, n_lines) : pick_warp_shape<T, 8>(p, n_lines, W);
  TPF_CHECK_ARG(s.TL > 0, "CCD axis of %lld points does not fit the line kernel's shared memory",
                (long long)p->n_pts);
  CcdArgs a{};
  a.f = f; a.d1 = d1; a.d2 = d2;
  a.outer = outer; a.inner = inner; a.n_lines = n_lines;
  a.n = (int)p->n_pts; a.n_rows = p->n_rows; a.C = p->C; a.P = p->P; a.H0 = p->H0; a.TL = s.TL;
  a.tl_shift = 0;
  while ((1 << a.tl_shift) < s.TL) ++a.tl_shift;
  a.LS = s.LS; a.FS = (contig || warp) ? s.FS : 0; a.nbuf = s.nbuf;
  a.n_tiles = (int)((n_lines + s.TL - 1) / s.TL);
  a.tab_total = TabLayout{p->C, p->H0}.total();
  a.tab = p->d_tab;
  a.tabT = std::is_same<T, double>::value ? (const void*)p->d_tab : (const void*)p->d_tabf;
  a.J = ((flags & TPF_CCD_APPLY_METRIC) && p->has_metric) ? p->d_J : nullptr;
  a.ovl = bcl ? 1 : 0;
  a.ovr = bcr ? 1 : 0;
  if (bcl) { a.bcl0 = bcl[0]; a.bcl1 = bcl[1]; }
  if (bcr) { a.bcr0 = bcr[0]; a.bcr1 = bcr[1]; }
  a.vd_rho = vd_rho;
  a.vd_drho = vd_drho;
  a.vd_out = vd_out;
  a.vd_accumulate = vd_accumulate;
  if (corrector) {
    a.cr_u = corrector->cr_u;
    a.cr_rho = corrector->cr_rho;
    a.cr_out = corrector->cr_out;
    a.cr_dt = corrector->cr_dt;
    a.cr_wall = corrector->cr_wall;
  }
  const bool per = (p->bc == TPF_BC_PERIODIC) && !a.ovl && !a.ovr;
  if (use_lane_kernel(p, n_lines, per, contig)) return launch_lane<T>(p, a, per, contig, stream);
  void (*kern)(CcdArgs);
  if (!warp) {
    if (per) kern = contig ? ccd_line_kernel<T, true, true> : ccd_line_kernel<T, true, false>;
    else kern = contig ? ccd_line_kernel<T, false, true> : ccd_line_kernel<T, false, false>;
  } else {
#define TPF_WARP_KERN(WW)                                                                               \
  if (per) kern = contig ? ccd_warp_kernel<T, true, true, 8, WW> : ccd_warp_kernel<T, true, false, 8, WW>; \
  else kern = contig ? ccd_warp_kernel<T, false, true, 8, WW> : ccd_warp_kernel<T, false, false, 8, WW>;
    if (W == 1) { TPF_WARP_KERN(1) }
    else if (W == 2) { TPF_WARP_KERN(2) }
    else { TPF_WARP_KERN(4) }
#undef TPF_WARP_KERN
  }
  auto launch = [&](const LaunchShape& sh) -> int {
    CcdArgs b = a;
    b.TL = sh.TL;
    b.tl_shift = 0;
    while ((1 << b.tl_shift) < sh.TL) ++b.tl_shift;
    b.FS = (contig || warp) ? sh.FS : 0;
    b.LS = sh.LS;
    b.nbuf = sh.nbuf;
    b.n_tiles = (int)((n_lines + sh.TL - 1) / sh.TL);
    TPF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    kern<<<sh.grid, warp ? 32 * W * sh.TL : sh.TL * p->P, sh.smem, stream>>>(b);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  };
  if (!warp) return launch(s);
  // Warp kernel: the launch shape (lines per block, tile buffers) is picked by
  // timing on the first call of each (line count, axis kind, boundary,
  // outputs, dtype) combination, like the lane kernel's; every shape gives
  // identical results (the lines are solved independently).
  const bool plain = a.d1 && a.d2 && !a.vd_out && !a.J && !a.cr_out;
  const uint64_t key = ((uint64_t)n_lines << 8) | (1ull << 7) | ((uint64_t)contig << 0) | ((uint64_t)per << 1) |
                       ((uint64_t)plain << 2) | ((uint64_t)(sizeof(T) == 8) << 3) | ((uint64_t)W << 4);
  auto it = p->lane_tuned.find(key);
  if (it != p->lane_tuned.end()) {
    const LaunchShape ts = warp_shape<T, 8>(p, n_lines, W, it->second.warps, it->second.nbuf);
    if (ts.TL > 0) return launch(ts);
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  TPF_CUDA_TRY(cudaStreamIsCapturing(stream, &cs));
  if (!p->autotune || cs != cudaStreamCaptureStatusNone || (a.vd_out && a.vd_accumulate) ||
      (a.cr_out && a.cr_out == a.cr_u))
    return launch(s);
  cudaEvent_t e0, e1;
  TPF_CUDA_TRY(cudaEventCreate(&e0));
  TPF_CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  LaunchShape bs = s;
  int st = TPF_OK;
  const int tls[4] = {8, 4, 2, 1};
  for (int ti = 0; ti < 4 && !st; ++ti) {
    for (int nbuf = 1; nbuf <= 2 && !st; ++nbuf) {
      const LaunchShape c = warp_shape<T, 8>(p, n_lines, W, tls[ti], nbuf);
      if (c.TL == 0) continue;
      if ((st = launch(c))) break;
      cudaEventRecord(e0, stream);
      for (int r = 0; r < 2 && !st; ++r) st = launch(c);
      cudaEventRecord(e1, stream);
      if (cudaEventSynchronize(e1) != cudaSuccess || st) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        bs = c;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  p->lane_tuned[key] = LaneShape_{bs.TL, bs.nbuf, 0};
  // the last candidate's results are in place and identical for every shape
  return TPF_OK;
}

// ---- FP32 line solves under FP64 iterative refinement (wall axes) ----------------
//
// d = K32(f) in FP32, then per refinement the residual of the full
// (N+1)-node CCD system, R = B f - A d, in FP64 (interior Eq-I / Eq-II rows,
// the one-sided closure rows at both walls, ccd_solver.py:11-22,408-465),
// and d += A^-1 R with the correction solved in FP32: the boundary rows are
// folded into the first / last interior rows (delta_0 = M_l delta_1 + R_0,
// ccd_solver_helpers.py:242-245), one thread runs the block-Thomas sweeps of
// a line with per-row factors, and the boundary corrections are recovered.

__device__ __forceinline__ float2 mv2f(const float* m, float a, float b) {
  return make_float2(m[0] * a + m[1] * b, m[2] * a + m[3] * b);
}

__global__ void ccd_cast_kernel(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void ccd_widen_kernel(int64_t n, const float* __restrict__ in, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// R = B f - A d at every node, FP64 arithmetic, FP32 storage
__global__ void ccd_resid_kernel(int64_t total, int64_t inner, int n, double h, const double* __restrict__ f,
                                 const double* __restrict__ d1, const double* __restrict__ d2,
                                 float* __restrict__ R1, float* __restrict__ R2) {
  const double a1h = kA1 / h, a2h2 = kA2 / (h * h), b1h = kB1 * h, b2h = kB2 / h;
  const double inv12h2 = 1.0 / (12.0 * h * h);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ln = e / inner;
    const int k = (int)(ln % n);
    const int64_t s = inner;
    double r1, r2;
    if (k == 0) {
      const double cI = (-23.0 / 6.0 * f[e] + 21.0 / 4.0 * f[e + s] - 1.5 * f[e + 2 * s] + 1.0 / 12.0 * f[e + 3 * s]) / h;
      const double cII = (45.0 * f[e] - 154.0 * f[e + s] + 214.0 * f[e + 2 * s] - 156.0 * f[e + 3 * s] +
                          61.0 * f[e + 4 * s] - 10.0 * f[e + 5 * s]) * inv12h2;
      r1 = cI - (d1[e] - (-1.5 * d1[e + s] + 1.5 * h * d2[e + s]));
      r2 = cII - d2[e];
    } else if (k == n - 1) {
      const double cI = (23.0 / 6.0 * f[e] - 21.0 / 4.0 * f[e - s] + 1.5 * f[e - 2 * s] - 1.0 / 12.0 * f[e - 3 * s]) / h;
      const double cII = (45.0 * f[e] - 154.0 * f[e - s] + 214.0 * f[e - 2 * s] - 156.0 * f[e - 3 * s] +
                          61.0 * f[e - 4 * s] - 10.0 * f[e - 5 * s]) * inv12h2;
      r1 = cI - (d1[e] - (-1.5 * d1[e - s] - 1.5 * h * d2[e - s]));
      r2 = cII - d2[e];
    } else {
      const double fm = f[e - s], f0 = f[e], fp = f[e + s];
      const double pm = d1[e - s], p0 = d1[e], pp = d1[e + s];
      const double qm = d2[e - s], q0 = d2[e], qp = d2[e + s];
      r1 = a1h * (fp - fm) - (kAlpha1 * (pm + pp) + p0 - b1h * (qp - qm));
      r2 = a2h2 * ((fm - 2.0 * f0) + fp) - (kBeta2 * (qm + qp) + q0 - b2h * (pp - pm));
    }
    R1[e] = (float)r1;
    R2[e] = (float)r2;
  }
}

// d += A^-1 R on every line (FP32 sweeps; R is overwritten by the forward sweep)
__global__ void ccd_corr_kernel(int64_t n_lines, int64_t inner, int n, float h, const float* __restrict__ fac,
                                float* R1, float* R2, double* d1, double* d2) {
  const int64_t L = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (L >= n_lines) return;
  const int64_t o = L / inner, i = L - o * inner;
  const int64_t base = o * (int64_t)n * inner + i;
  const int64_t s = inner;
  const int nr = n - 2;
  const float La[4] = {(float)kAlpha1, (float)kB1 * h, (float)kB2 / h, (float)kBeta2};
  const float Ua[4] = {(float)kAlpha1, -(float)kB1 * h, -(float)kB2 / h, (float)kBeta2};
  const float Ml[4] = {-1.5f, 1.5f * h, 0.0f, 0.0f};
  const float Mr[4] = {-1.5f, -1.5f * h, 0.0f, 0.0f};
  const float r0a = R1[base], r0b = R2[base];
  const float rNa = R1[base + (int64_t)(n - 1) * s], rNb = R2[base + (int64_t)(n - 1) * s];
  float ya = 0.0f, yb = 0.0f;
  for (int j = 0; j < nr; ++j) {
    const int64_t e = base + (int64_t)(j + 1) * s;
    float ra = R1[e], rb = R2[e];
    if (j == 0) {
      const float2 q = mv2f(La, r0a, r0b);
      ra -= q.x;
      rb -= q.y;
    }
    if (j == nr - 1) {
      const float2 q = mv2f(Ua, rNa, rNb);
      ra -= q.x;
      rb -= q.y;
    }
    const float* lf = fac + 12 * j;
    const float2 q = mv2f(lf, ya, yb);
    ya = ra - q.x;
    yb = rb - q.y;
    R1[e] = ya;
    R2[e] = yb;
  }
  float xa = 0.0f, xb = 0.0f, x1a = 0.0f, x1b = 0.0f, xla = 0.0f, xlb = 0.0f;
  for (int j = nr - 1; j >= 0; --j) {
    const int64_t e = base + (int64_t)(j + 1) * s;
    const float* pm = fac + 12 * j + 4;
    const float* hm = pm + 4;
    const float2 py = mv2f(pm, R1[e], R2[e]);
    const float2 hx = mv2f(hm, xa, xb);
    xa = py.x - hx.x;
    xb = py.y - hx.y;
    d1[e] += (double)xa;
    d2[e] += (double)xb;
    if (j == nr - 1) { xla = xa; xlb = xb; }
    if (j == 0) { x1a = xa; x1b = xb; }
  }
  const float2 b0 = mv2f(Ml, x1a, x1b);
  const float2 bN = mv2f(Mr, xla, xlb);
  d1[base] += (double)(b0.x + r0a);
  d2[base] += (double)(b0.y + r0b);
  d1[base + (int64_t)(n - 1) * s] += (double)(bN.x + rNa);
  d2[base + (int64_t)(n - 1) * s] += (double)(bN.y + rNb);
}

// per-row factors of the folded wall system (the recurrence of build_tables)
int refine_factors(const tpf_ccd_plan* p) {
  if (p->d_rfac) return TPF_OK;
  const double h = p->h;
  const int nr = p->n_rows;
  const M2 L = {kAlpha1, kB1 * h, kB2 / h, kBeta2};
  const M2 U = {kAlpha1, -kB1 * h, -kB2 / h, kBeta2};
  const M2 Ml = {-1.5, 1.5 * h, 0.0, 0.0};
  const M2 Mr = {-1.5, -1.5 * h, 0.0, 0.0};
  std::vector<float> fac((size_t)12 * nr);
  M2 LUp = eye();
  for (int j = 0; j < nr; ++j) {
    M2 D = eye();
    if (j == 0) D = add(D, mul(L, Ml));
    if (j == nr - 1) D = add(D, mul(U, Mr));
    M2 Lf = {0, 0, 0, 0}, LU;
    if (j == 0) LU = D;
    else {
      Lf = mul(L, inv(LUp));
      LU = sub(D, mul(Lf, U));
    }
    const double dt = det(LU);
    if (!std::isfinite(dt) || std::fabs(dt) < 1e-300) {
      tpf::set_error("CCD block-tridiagonal factorization encountered a singular pivot at block %d", j);
      return TPF_ESINGULAR;
    }
    const M2 Pm = inv(LU);
    const M2 Hm = (j < nr - 1) ? mul(Pm, U) : M2{0, 0, 0, 0};
    for (int q = 0; q < 4; ++q) {
      fac[12 * j + q] = (float)Lf[q];
      fac[12 * j + 4 + q] = (float)Pm[q];
      fac[12 * j + 8 + q] = (float)Hm[q];
    }
    LUp = LU;
  }
  float* d = nullptr;
  if (cudaMalloc(&d, fac.size() * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    tpf::set_error("cudaMalloc of the refinement factors failed");
    return TPF_ECUDA;
  }
  if (cudaMemcpy(d, fac.data(), fac.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d);
    tpf::set_error("cudaMemcpy of the refinement factors failed");
    return TPF_ECUDA;
  }
  p->d_rfac = d;
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
  // chunk length = rows per lane of the warp kernel (8; 1, 2 or 4 warps per
  // line up to 1024 rows); longer lines use the shared-memory chunk kernel
  // with C = ceil(n_rows / 32)
  p->C = p->n_rows <= 1024 ? 8 : (p->n_rows + 31) / 32;
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
  {
    const std::vector<double>& lt = p->ltab_host;
    std::vector<float> ltf(lt.begin(), lt.end());
    p->ltab_total = (int)lt.size();
    if (cudaMalloc(&p->d_ltab, lt.size() * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&p->d_ltabf, lt.size() * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(p->d_ltab, lt.data(), lt.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_ltabf, ltf.data(), ltf.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      tpf::set_error("allocation / copy of the CCD lane table failed");
      cudaFree(p->d_tab);
      cudaFree(p->d_tabf);
      cudaFree(p->d_ltab);
      cudaFree(p->d_ltabf);
      delete p;
      return TPF_ECUDA;
    }
  }
  *out = p;
  return TPF_OK;
}

int tpf_ccd_plan_set_autotune(tpf_ccd_plan* p, int enable) {
  TPF_CHECK_ARG(p != nullptr, "plan is NULL");
  p->autotune = enable != 0;
  if (!enable) p->lane_tuned.clear();
  return TPF_OK;
}

int tpf_ccd_plan_destroy(tpf_ccd_plan* p) {
  if (!p) return TPF_OK;
  cudaFree(p->d_tab);
  cudaFree(p->d_tabf);
  cudaFree(p->d_ltab);
  cudaFree(p->d_ltabf);
  cudaFree(p->d_J);
  cudaFree(p->d_rfac);
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

int tpf_ccd_apply_refined(const tpf_ccd_plan* p64, const tpf_ccd_plan* p32, int64_t outer, int64_t inner,
                          const double* f, double* d1, double* d2, int refinements, float* work, void* stream) {
  TPF_CHECK_ARG(p64 && p32 && f && d1 && d2 && work, "NULL argument");
  TPF_CHECK_ARG(p64->dtype == TPF_F64 && p32->dtype == TPF_F32, "plans must be FP64 and FP32");
  TPF_CHECK_ARG(p64->bc == TPF_BC_WALL && p32->bc == TPF_BC_WALL,
                "iterative refinement of the CCD line solves covers wall axes");
  TPF_CHECK_ARG(p64->n_pts == p32->n_pts && p64->h == p32->h, "the FP64 and FP32 plans differ");
  TPF_CHECK_ARG(outer >= 0 && inner >= 1, "invalid line decomposition");
  TPF_CHECK_ARG(refinements >= 0 && refinements <= 8, "refinements must be in [0, 8]");
  TPF_CHECK_ARG(f != d1 && f != d2 && d1 != d2, "f, d1 and d2 must be distinct");
  const int64_t n_lines = outer * inner;
  if (n_lines == 0) return TPF_OK;
  int st = refine_factors(p64);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = (int)p64->n_pts;
  const int64_t total = n_lines * n;
  float* f32 = work;
  float* a32 = work + total;
  float* b32 = work + 2 * total;
  float* R1 = work + 3 * total;
  float* R2 = work + 4 * total;
  const int eb = (int)std::min<int64_t>((total + 255) / 256, 8 * 148 * 4);
  ccd_cast_kernel<<<eb, 256, 0, s>>>(total, f, f32);
  TPF_CUDA_TRY(cudaGetLastError());
  if ((st = launch_ccd<float>(p32, outer, inner, f32, a32, b32, nullptr, nullptr, 0, s))) return st;
  ccd_widen_kernel<<<eb, 256, 0, s>>>(total, a32, d1);
  ccd_widen_kernel<<<eb, 256, 0, s>>>(total, b32, d2);
  for (int r = 0; r < refinements; ++r) {
    ccd_resid_kernel<<<eb, 256, 0, s>>>(total, inner, n, p64->h, f, d1, d2, R1, R2);
    ccd_corr_kernel<<<(int)((n_lines + 127) / 128), 128, 0, s>>>(n_lines, inner, n, (float)p64->h, p64->d_rfac, R1,
                                                                 R2, d1, d2);
  }
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int tpf_ccd_apply_vd(const tpf_ccd_plan* p, int64_t outer, int64_t inner, const void* f, const void* rho,
                     const void* drho, void* out, int accumulate, int flags, void* stream) {
  TPF_CHECK_ARG(p != nullptr, "plan is NULL");
  TPF_CHECK_ARG(outer >= 0 && inner >= 1, "invalid line decomposition");
  TPF_CHECK_ARG(f && rho && drho && out, "NULL argument");
  TPF_CHECK_ARG(!(flags & TPF_CCD_APPLY_METRIC) || p->has_metric, "metric requested but not set");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->dtype == TPF_F64)
    return launch_ccd<double>(p, outer, inner, f, nullptr, nullptr, nullptr, nullptr, flags, s, rho, drho, out,
                              accumulate);
  return launch_ccd<float>(p, outer, inner, f, nullptr, nullptr, nullptr, nullptr, flags, s, rho, drho, out,
                           accumulate);
}

int tpf_ccd_apply_corrector(const tpf_ccd_plan* p, int64_t outer, int64_t inner, const void* pres,
                            const void* u_star, const void* rho, double dt, void* u_out, int flags, void* stream) {
  TPF_CHECK_ARG(p != nullptr, "plan is NULL");
  TPF_CHECK_ARG(outer >= 0 && inner >= 1, "invalid line decomposition");
  TPF_CHECK_ARG(pres && u_star && rho && u_out, "NULL argument");
  TPF_CHECK_ARG(!(flags & TPF_CCD_APPLY_METRIC) || p->has_metric, "metric requested but not set");
  CcdArgs cr{};
  cr.cr_u = u_star;
  cr.cr_rho = rho;
  cr.cr_out = u_out;
  cr.cr_dt = dt;
  cr.cr_wall = (p->bc == TPF_BC_WALL) ? 1 : 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->dtype == TPF_F64)
    return launch_ccd<double>(p, outer, inner, pres, nullptr, nullptr, nullptr, nullptr, flags, s, nullptr, nullptr,
                              nullptr, 0, &cr);
  return launch_ccd<float>(p, outer, inner, pres, nullptr, nullptr, nullptr, nullptr, flags, s, nullptr, nullptr,
                           nullptr, 0, &cr);
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

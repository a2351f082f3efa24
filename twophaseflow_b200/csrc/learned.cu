// Network-preconditioned flexible CG for the variable-density PPE.
//
// Solves the same control-volume-weighted SPD system as the CG route of
// PPESolverFVMMatrixFree (S p = -W rhs, pinned node removed), with a
// preconditioner that is a trained U-Net (unet.cu) applied to the
// Jacobi-scaled residual, optionally followed by damped-Jacobi smoothing:
//
//   r~ = D^-1/2 r / s,  s = rms(D^-1/2 r),   c~ = ln(rho_max / rho) / ln(1000)
//   z  = s D^-1/2 UNet(r~, c~)               (BF16 network, FP32 accumulation)
//   z <- z + omega D^-1 (r - S z)             (`smooth` times)
//
// The preconditioner is not a fixed linear map, so the outer iteration is
// flexible CG (Notay's truncated FCG with one stored direction): each new
// direction is A-orthogonalised against the previous one.  All four inner
// products an iteration needs come from one fused stencil+reduction pass
// (S symmetric: (p', S z) = (S p', z)), vectors and scalars stay in FP64 on
// the device, and one iteration is replayed as a CUDA graph.  Convergence is
// checked on the true residual b - S x at the end; when the residual stops
// falling the solve continues with the plain Jacobi PCG kernel from the
// current iterate.
//
// The reference has no learned preconditioner; parity is "equals the FP64
// solution of the same system within the stated tolerance".
#include "tpf_common.cuh"
#include "ppe_view.cuh"
#include "tc_sm100.cuh"
#include "gmres.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

typedef __nv_bfloat16 bf16;

namespace {

constexpr int kRedBlocks = 296;   // 2 x SM count, fixed for deterministic reductions
constexpr int kRedThreads = 256;

struct LGrid {
  int n0, n1, ndof, pin;
  int H, W;            // network image (multiple of 8): fine nodes, or aggregates when b > 1
  int b, nc0, nc1;     // aggregate size and coarse grid (b = 1: the network runs on the fine grid)
  const double* s0;
  const double* s1;
  const double* dinvS;
  const double* dv0;
  const double* dv1;
  const double* dcis;  // coarse D_c^-1/2 (b > 1)
  const float* featc;  // coarse density feature (b > 1)
};

constexpr int kMaxWin = 8;   // stored directions of the truncated flexible CG

struct FcgState {
  double bb, rr, rdr;
  double s, inv_s;       // network input scale
  double delta[kMaxWin]; // (p_j, S p_j) of the stored directions
  double beta[kMaxWin];  // projections of the new preconditioned residual
  double alpha;
  int count;             // stored directions in use (0 after a restart)
  int head;              // ring slot of the newest direction
  int used;              // directions projected out this iteration
  int slot;              // ring slot receiving this iteration's direction
  int win;               // window length m
  double tol2;
  double sc, inv_sc;      // coarse network input scale (two-level mode)
  long long iters;
  int done;
  int restarts;
};

__device__ __forceinline__ double s_apply(const LGrid& g, const double* __restrict__ z, int idx, int i0, int i1) {
  const double sm0 = (i0 > 0) ? g.s0[idx - g.n1] : 0.0;
  const double sp0 = g.s0[idx];
  const double sm1 = (i1 > 0) ? g.s1[idx - 1] : 0.0;
  const double sp1 = g.s1[idx];
  double off = 0.0;
  if (i0 > 0) off += sm0 * z[idx - g.n1];
  if (i0 < g.n0 - 1) off += sp0 * z[idx + g.n1];
  if (i1 > 0) off += sm1 * z[idx - 1];
  if (i1 < g.n1 - 1) off += sp1 * z[idx + 1];
  return (sm0 + sp0 + sm1 + sp1) * z[idx] - off;
}

template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* part) {
  __shared__ double scratch[NV * 32];
  tpf::block_sum<NV>(v, scratch);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) part[k * gridDim.x + blockIdx.x] = v[k];
  }
}

// sum of the per-block partials (one block, fixed order -> deterministic)
template <int NV>
__device__ __forceinline__ void reduce_partials(const double* part, int nb, double (&out)[NV]) {
  __shared__ double scratch[NV * 32];
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double a = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) a += part[k * nb + i];
    v[k] = a;
  }
  tpf::block_sum<NV>(v, scratch);
#pragma unroll
  for (int k = 0; k < NV; ++k) out[k] = v[k];
}

__device__ __forceinline__ void set_scale(FcgState* st, double rdr, int ndof) {
  const double s = sqrt(rdr / ndof);
  st->s = s;
  st->inv_s = (s > 0.0) ? 1.0 / s : 0.0;
}

// b = -W rhs (pin 0), x = x0 (pin 0)
__global__ void fcg_init_kernel(LGrid g, const double* rhs, const double* x0, double* b, double* x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    b[i] = (i == g.pin) ? 0.0 : -(rhs[i] * g.dv0[i0] * g.dv1[i1]);
    x[i] = (x0 && i != g.pin) ? x0[i] : 0.0;
  }
}

// r = b - S x (pin 0); partials: r.r, r.r dinvS, b.b
__global__ void __launch_bounds__(kRedThreads) fcg_residual_kernel(LGrid g, const double* b, const double* x,
                                                                   double* r, double* part) {
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    const double ri = (i == g.pin) ? 0.0 : b[i] - s_apply(g, x, i, i0, i1);
    r[i] = ri;
    v[0] += ri * ri;
    v[1] += ri * ri * g.dinvS[i];
    v[2] += b[i] * b[i];
  }
  block_partials<3>(v, part);
}

// first == 1: start of a solve (sets ||b||, the tolerance, the counters);
// first == 0: true-residual check / restart.
__global__ void fcg_start_kernel(const double* part, int nb, int ndof, FcgState* st, double tol, int first, int win) {
  double v[3];
  reduce_partials<3>(part, nb, v);
  if (threadIdx.x == 0) {
    if (first) {
      st->bb = v[2];
      st->tol2 = tol * tol * v[2];
      st->iters = 0;
      st->restarts = 0;
      st->win = win;
    } else {
      st->restarts += 1;
    }
    st->rr = v[0];
    st->rdr = v[1];
    set_scale(st, v[1], ndof);
    st->count = 0;
    st->head = -1;
    st->used = 0;
    st->alpha = 0.0;
    st->done = (v[0] <= st->tol2) ? 1 : 0;
  }
}

// network input: channel 0 = D^-1/2 r / s, 1 = c~, 2 / 3 = the Jacobi-scaled
// couplings to the next row / column (D^-1/2 S D^-1/2 = I - couplings), 4..15 = 0
__device__ __forceinline__ void fine_coupl(const LGrid& g, int i, int i0, int i1, float& a0, float& a1) {
  a0 = (i0 + 1 < g.n0) ? (float)(g.s0[i] * sqrt(g.dinvS[i] * g.dinvS[i + g.n1])) : 0.f;
  a1 = (i1 + 1 < g.n1) ? (float)(g.s1[i] * sqrt(g.dinvS[i] * g.dinvS[i + 1])) : 0.f;
}

__device__ __forceinline__ uint4 pack4bf(float c0, float c1, float c2, float c3) {
  uint4 v = make_uint4(0, 0, 0, 0);
  __nv_bfloat162 h0 = __floats2bfloat162_rn(c0, c1), h1 = __floats2bfloat162_rn(c2, c3);
  v.x = *reinterpret_cast<uint32_t*>(&h0);
  v.y = *reinterpret_cast<uint32_t*>(&h1);
  return v;
}

__global__ void fcg_pack_kernel(LGrid g, const double* r, const float* feat, const FcgState* st, bf16* xin) {
  tpf::chain_begin();
  tpf::tc::pdl_trigger();
  if (st->done) return;
  const int Wp = g.W + 2;
  const long long P = (long long)(g.H + 2) * Wp;
  const float inv_s = (float)st->inv_s;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int yy = (int)(q / Wp), xx = (int)(q - (long long)yy * Wp);
    const int y = yy - 1, x = xx - 1;
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
    if (y >= 0 && y < g.n0 && x >= 0 && x < g.n1) {
      const int i = y * g.n1 + x;
      c0 = (float)(r[i] * sqrt(g.dinvS[i])) * inv_s;
      c1 = feat[i];
      fine_coupl(g, i, y, x, c2, c3);
    }
    uint4* o = reinterpret_cast<uint4*>(xin + q * 16);
    o[0] = pack4bf(c0, c1, c2, c3);
    o[1] = make_uint4(0, 0, 0, 0);
  }
  tpf::chain_end();
}

// z = s D^-1/2 y (pin 0)
__global__ void fcg_unpack_kernel(LGrid g, const float* y, const FcgState* st, double* z) {
  tpf::chain_begin();
  if (st->done) return;
  const double s = st->s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    z[i] = (i == g.pin) ? 0.0 : s * sqrt(g.dinvS[i]) * (double)y[(size_t)i0 * g.W + i1];
  }
  tpf::chain_end();
}

// one damped-Jacobi update of a node, z + omega D^-1 (r - S z), from its
// value, its four neighbours' values and couplings (h*: whether the
// neighbour exists); shared by the single-sweep and the blocked smoother so
// that both round identically
__device__ __forceinline__ double jacobi_node(double zc, double zm0, double zp0, double zm1, double zp1, double sm0,
                                              double sp0, double sm1, double sp1, bool h0m, bool h0p, bool h1m,
                                              bool h1p, double dinv, double rr, double omega) {
  double off = 0.0;
  if (h0m) off += sm0 * zm0;
  if (h0p) off += sp0 * zp0;
  if (h1m) off += sm1 * zm1;
  if (h1p) off += sp1 * zp1;
  const double sz = (sm0 + sp0 + sm1 + sp1) * zc - off;
  return zc + omega * dinv * (rr - sz);
}

// the prolongated coarse correction plus the pre-smoothing term at node j:
// z2 = omega D^-1 r + P (s_c D_c^-1/2 y) (pin 0); two-level mode
__device__ __forceinline__ double prolong_value(const LGrid& g, const float* y, const double* r, double omega,
                                                double sc, int j, int j0, int j1) {
  if (j == g.pin) return 0.0;
  const int J0 = j0 / g.b, J1 = j1 / g.b;
  return omega * g.dinvS[j] * r[j] + sc * g.dcis[J0 * g.nc1 + J1] * (double)y[(size_t)J0 * g.W + J1];
}

// zout = zin + omega D^-1 (r - S zin) (pin 0)
__global__ void fcg_smooth_kernel(LGrid g, const double* zin, const double* r, double omega, const FcgState* st,
                                  double* zout) {
  tpf::chain_begin();
  if (st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    if (i == g.pin) {
      zout[i] = 0.0;
      continue;
    }
    const bool h0m = i0 > 0, h0p = i0 < g.n0 - 1, h1m = i1 > 0, h1p = i1 < g.n1 - 1;
    zout[i] = jacobi_node(zin[i], h0m ? zin[i - g.n1] : 0.0, h0p ? zin[i + g.n1] : 0.0, h1m ? zin[i - 1] : 0.0,
                          h1p ? zin[i + 1] : 0.0, h0m ? g.s0[i - g.n1] : 0.0, g.s0[i], h1m ? g.s1[i - 1] : 0.0,
                          g.s1[i], h0m, h0p, h1m, h1p, g.dinvS[i], r[i], omega);
  }
  tpf::chain_end();
}

// k <= kSmK damped-Jacobi sweeps in one pass (temporal blocking): a CTA loads
// z, r, D^-1 and the couplings of its kSmTY x kSmTX tile plus a kSmK-node
// halo into shared memory, sweeps k times over a region that shrinks by one
// node per sweep, and writes the tile; each node's update is the single
// sweep's (jacobi_node), so the result equals k single sweeps bit for bit
constexpr int kSmTX = 32, kSmTY = 16, kSmK = 4;
constexpr int kSmW = kSmTX + 2 * kSmK, kSmH = kSmTY + 2 * kSmK;

constexpr int kSmThreads = 512;

// yprol non-null (two-level mode): the sweeps start from the prolongated
// correction z2 = omega D^-1 r + P (s_c D_c^-1/2 yprol) instead of zin, so the
// first sweep is the prolongation sweep of prolong_smooth_kernel
__global__ void __launch_bounds__(kSmThreads, 2) smooth_block_kernel(LGrid g, const double* zin, const float* yprol,
                                                                     const double* r, double omega, int k,
                                                                     const FcgState* st, double* zout) {
  tpf::chain_begin();
  if (st->done) return;
  const double sc = yprol ? st->sc : 0.0;
  // only z goes through shared memory; each thread keeps r, D^-1 and the four
  // couplings of its own kPer nodes (e = tid + kSmThreads j of the tile with
  // halo) in registers for all k sweeps and holds its last updates for the store
  __shared__ double sz[2][kSmH][kSmW];
  constexpr int kPer = (kSmH * kSmW + kSmThreads - 1) / kSmThreads;
  const int tiles1 = (g.n1 + kSmTX - 1) / kSmTX;
  const int base0 = (int)(blockIdx.x / tiles1) * kSmTY - kSmK;
  const int base1 = (int)(blockIdx.x % tiles1) * kSmTX - kSmK;
  double lz[kPer], lr[kPer], ld[kPer], m0[kPer], p0[kPer], m1[kPer], p1[kPer];
  // bit 0 in the domain, 1 pinned, 2..5 neighbours -0 +0 -1 +1 exist,
  // bits 8..15 the tile column, 16..23 the tile row
  unsigned flags[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int e = threadIdx.x + j * kSmThreads;
    const int a = e / kSmW, c = e - (e / kSmW) * kSmW;
    const int i0 = base0 + a, i1 = base1 + c;
    const bool in = e < kSmH * kSmW && i0 >= 0 && i0 < g.n0 && i1 >= 0 && i1 < g.n1;
    const int i = in ? i0 * g.n1 + i1 : 0;
    const bool h0m = in && i0 > 0, h0p = in && i0 < g.n0 - 1, h1m = in && i1 > 0, h1p = in && i1 < g.n1 - 1;
    flags[j] = (in ? 1u : 0u) | ((in && i == g.pin) ? 2u : 0u) | (h0m ? 4u : 0u) | (h0p ? 8u : 0u) |
               (h1m ? 16u : 0u) | (h1p ? 32u : 0u) | ((unsigned)c << 8) | ((unsigned)a << 16);
    lz[j] = in ? (yprol ? prolong_value(g, yprol, r, omega, sc, i, i0, i1) : zin[i]) : 0.0;
    lr[j] = in ? r[i] : 0.0;
    ld[j] = in ? g.dinvS[i] : 0.0;
    m0[j] = h0m ? g.s0[i - g.n1] : 0.0;
    p0[j] = in ? g.s0[i] : 0.0;
    m1[j] = h1m ? g.s1[i - 1] : 0.0;
    p1[j] = in ? g.s1[i] : 0.0;
  }
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int e = threadIdx.x + j * kSmThreads;
    if (e < kSmH * kSmW) {
      const int a = (int)((flags[j] >> 16) & 255u), c = (int)((flags[j] >> 8) & 255u);
      sz[0][a][c] = lz[j];
      sz[1][a][c] = 0.0;
    }
  }
  __syncthreads();
  int cur = 0;
  for (int sweep = 1; sweep <= k; ++sweep) {
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const int a = (int)((flags[j] >> 16) & 255u), c = (int)((flags[j] >> 8) & 255u);
      if (!(flags[j] & 1u) || a < sweep || a >= kSmH - sweep || c < sweep || c >= kSmW - sweep) continue;
      const double v =
          (flags[j] & 2u)
              ? 0.0
              : jacobi_node(sz[cur][a][c], sz[cur][a - 1][c], sz[cur][a + 1][c], sz[cur][a][c - 1],
                            sz[cur][a][c + 1], m0[j], p0[j], m1[j], p1[j], (flags[j] & 4u) != 0,
                            (flags[j] & 8u) != 0, (flags[j] & 16u) != 0, (flags[j] & 32u) != 0, ld[j], lr[j], omega);
      sz[cur ^ 1][a][c] = v;
      lz[j] = v;
    }
    cur ^= 1;
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int a = (int)((flags[j] >> 16) & 255u), c = (int)((flags[j] >> 8) & 255u);
    if (!(flags[j] & 1u) || a < kSmK || a >= kSmK + kSmTY || c < kSmK || c >= kSmK + kSmTX) continue;
    zout[(base0 + a) * g.n1 + base1 + c] = lz[j];
  }
  tpf::chain_end();
}

// w = S z (pin 0); partials (z, Q_j) and (P_j, r) for the stored directions,
// (z, r), (z, w): everything the step needs in one pass (S is symmetric, so
// (P_j, S z) = (Q_j, z) and A-orthogonality gives (p, S p) without a second pass)
template <int M>
__global__ void __launch_bounds__(kRedThreads) fcg_sdot_kernel(LGrid g, const double* z, const double* r,
                                                               const double* P, const double* Q, double* w,
                                                               const FcgState* st, double* part) {
  if (st->done) return;
  constexpr int NV = 2 * M + 2;
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  const int cnt = st->count;
  const size_t nd = (size_t)g.ndof;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    const double wi = (i == g.pin) ? 0.0 : s_apply(g, z, i, i0, i1);
    w[i] = wi;
    const double zi = z[i], ri = r[i];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      if (j < cnt) {
        v[j] += zi * Q[j * nd + i];
        v[M + j] += P[j * nd + i] * ri;
      }
    }
    v[2 * M] += zi * ri;
    v[2 * M + 1] += zi * wi;
  }
  block_partials<NV>(v, part);
}

// beta_j, alpha and the ring bookkeeping of the truncated flexible CG step
template <int M>
__global__ void fcg_coef_kernel(const double* part, int nb, FcgState* st) {
  if (st->done) return;
  constexpr int NV = 2 * M + 2;
  double v[NV];
  reduce_partials<NV>(part, nb, v);
  if (threadIdx.x == 0) {
    const int cnt = st->count;
    const double zr = v[2 * M], zw = v[2 * M + 1];
    double pq = zw, pr = zr;
    for (int j = 0; j < M; ++j) {
      const double b = (j < cnt && st->delta[j] > 0.0) ? v[j] / st->delta[j] : 0.0;
      st->beta[j] = b;
      pq -= b * v[j];
      pr -= b * v[M + j];
    }
    int used = cnt;
    if (!(pq > 1e-12 * zw) || !(pq > 0.0)) {   // lost A-orthogonality: restart the window
      used = 0;
      pq = zw;
      pr = zr;
      for (int j = 0; j < M; ++j) st->beta[j] = 0.0;
    }
    const int win = st->win < 1 ? 1 : (st->win > M ? M : st->win);
    // new direction: slot 0 after a restart, else the next ring slot (a full
    // window overwrites its oldest direction)
    const int slot = (used == 0) ? 0 : (st->head + 1) % win;
    st->used = used;
    st->slot = slot;
    st->alpha = (pq > 0.0) ? pr / pq : 0.0;
    st->delta[slot] = pq;
    st->head = slot;
    st->count = (used + 1 < win) ? used + 1 : win;
  }
}

// p = z - sum_j beta_j P_j, q = w - sum_j beta_j Q_j -> ring slot; x += alpha p,
// r -= alpha q; partials r.r, r.r dinvS
template <int M>
__global__ void __launch_bounds__(kRedThreads) fcg_update_kernel(LGrid g, const double* z, const double* w,
                                                                 double* P, double* Q, double* x, double* r,
                                                                 const FcgState* st, double* part) {
  if (st->done) return;
  const double alpha = st->alpha;
  const int used = st->used, slot = st->slot;
  double beta[M];
#pragma unroll
  for (int j = 0; j < M; ++j) beta[j] = st->beta[j];
  const size_t nd = (size_t)g.ndof;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    double pi = z[i], qi = w[i];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      if (j < used) {
        pi -= beta[j] * P[j * nd + i];
        qi -= beta[j] * Q[j * nd + i];
      }
    }
    P[slot * nd + i] = pi;
    Q[slot * nd + i] = qi;
    x[i] += alpha * pi;
    const double ri = r[i] - alpha * qi;
    r[i] = ri;
    v[0] += ri * ri;
    v[1] += ri * ri * g.dinvS[i];
  }
  block_partials<2>(v, part);
}

__global__ void fcg_finish_iter_kernel(const double* part, int nb, int ndof, FcgState* st) {
  if (st->done) return;
  double v[2];
  reduce_partials<2>(part, nb, v);
  if (threadIdx.x == 0) {
    st->rr = v[0];
    st->rdr = v[1];
    set_scale(st, v[1], ndof);
    st->iters += 1;
    if (v[0] <= st->tol2) st->done = 1;
  }
}

// c~ = clamp(ln(rho_max / rho) / ln(1000), 0, 1) from rho; rho_max by an integer max of the float bits
__global__ void rho_max_kernel(int n, const double* rho, unsigned long long* mx) {
  unsigned long long m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = rho[i] > 0.0 ? rho[i] : 0.0;
    m = max(m, (unsigned long long)__double_as_longlong(v));
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, m);
}

__global__ void feature_kernel(int n, const double* rho, const unsigned long long* mx, float* feat) {
  const double rmax = __longlong_as_double((long long)*mx);
  const double inv_l = 1.0 / log(1000.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double c = (rho[i] > 0.0) ? log(rmax / rho[i]) * inv_l : 1.0;
    c = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
    feat[i] = (float)c;
  }
}

// training pair from an error field e (pin 0): r = S e,
// in2 = (D^-1/2 r / s, c~), target = D^1/2 e / s on the network image (zero padding)
__global__ void __launch_bounds__(kRedThreads) pair_residual_kernel(LGrid g, const double* e, double* r,
                                                                    double* part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    const double ri = (i == g.pin) ? 0.0 : s_apply(g, e, i, i0, i1);
    r[i] = ri;
    v[0] += ri * ri * g.dinvS[i];
  }
  block_partials<1>(v, part);
}

__global__ void pair_write_kernel(LGrid g, const double* e, const double* r, const float* feat, const double* part,
                                  int nb, float* in, float* target) {
  __shared__ double s_inv;
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int i = 0; i < nb; ++i) a += part[i];
    const double s = sqrt(a / g.ndof);
    s_inv = (s > 0.0) ? 1.0 / s : 0.0;
  }
  __syncthreads();
  const double inv_s = s_inv;
  const long long n = (long long)g.H * g.W;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(q / g.W), x = (int)(q - (long long)y * g.W);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, t = 0.f;
    if (y < g.n0 && x < g.n1) {
      const int i = y * g.n1 + x;
      const double d = sqrt(g.dinvS[i]);
      a0 = (float)(r[i] * d * inv_s);
      a1 = feat[i];
      fine_coupl(g, i, y, x, a2, a3);
      t = (i == g.pin) ? 0.f : (float)(e[i] / d * inv_s);
    }
    in[4 * q] = a0;
    in[4 * q + 1] = a1;
    in[4 * q + 2] = a2;
    in[4 * q + 3] = a3;
    target[q] = t;
  }
}

__global__ void copy_x_kernel(int n, int pin, const double* x, double* p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = (i == pin) ? 0.0 : x[i];
}

// scale of an arbitrary residual (preconditioner applied outside a solve)
__global__ void __launch_bounds__(kRedThreads) rscale_partials_kernel(LGrid g, const double* r, double* part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x)
    v[0] += r[i] * r[i] * g.dinvS[i];
  block_partials<1>(v, part);
}

__global__ void rscale_finish_kernel(const double* part, int nb, int ndof, FcgState* st) {
  double v[1];
  reduce_partials<1>(part, nb, v);
  if (threadIdx.x == 0) {
    set_scale(st, v[0], ndof);
    st->done = 0;
  }
}

// ---- two-level mode: the network solves the aggregated coarse problem ---------------
//
// Aggregates are b x b blocks of fine nodes; R sums a block, P copies the coarse
// value back to its nodes.  The coarse operator A_c = R S P is a 5-point stencil
// whose couplings are the fine couplings crossing aggregate boundaries; only its
// diagonal D_c is formed (for the Jacobi-type scaling of the network input).
// One preconditioner application is a two-grid V(1, smooth) cycle:
//   z1 = w D^-1 r,  r1 = r - S z1,  z2 = z1 + P (s_c D_c^-1/2 UNet(D_c^-1/2 R r1 / s_c, c~_c)),
//   z  = z2 + w D^-1 (r - S z2)  (smooth times)

// D_c (sum of the fine couplings crossing the aggregate's boundary) and the
// Galerkin couplings to the aggregate below / to the right, gathered per
// aggregate in a fixed order (deterministic, no atomics)
__global__ void coarse_operator_kernel(LGrid g, double* dc, double* c0, double* c1) {
  const int nc = g.nc0 * g.nc1;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    const int I0 = I / g.nc1, I1 = I - I0 * g.nc1;
    const int a0 = I0 * g.b, a1 = I1 * g.b;
    const int e0 = min(g.n0, a0 + g.b), e1 = min(g.n1, a1 + g.b);
    double d = 0.0, down = 0.0, right = 0.0;
    for (int i0 = a0; i0 < e0; ++i0)
      for (int i1 = a1; i1 < e1; ++i1) {
        const int i = i0 * g.n1 + i1;
        if (i0 == a0 && i0 > 0) d += g.s0[i - g.n1];
        if (i0 == e0 - 1 && i0 + 1 < g.n0) {
          d += g.s0[i];
          down += g.s0[i];
        }
        if (i1 == a1 && i1 > 0) d += g.s1[i - 1];
        if (i1 == e1 - 1 && i1 + 1 < g.n1) {
          d += g.s1[i];
          right += g.s1[i];
        }
      }
    dc[I] = d;
    c0[I] = down;
    c1[I] = right;
  }
}

// D_c^-1/2 and the aggregate-mean density feature
__global__ void coarse_setup_kernel(LGrid g, const double* dc, const float* feat, double* dcis, float* featc) {
  const int nc = g.nc0 * g.nc1;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    dcis[I] = dc[I] > 0.0 ? 1.0 / sqrt(dc[I]) : 0.0;
    const int I0 = I / g.nc1, I1 = I - I0 * g.nc1;
    float acc = 0.f;
    int cnt = 0;
    for (int a0 = I0 * g.b; a0 < min(g.n0, (I0 + 1) * g.b); ++a0)
      for (int a1 = I1 * g.b; a1 < min(g.n1, (I1 + 1) * g.b); ++a1) {
        acc += feat[a0 * g.n1 + a1];
        ++cnt;
      }
    featc[I] = cnt ? acc / cnt : 0.f;
  }
}

// r1 = r - S (w D^-1 r), pin 0 (the pre-smoothing sweep from a zero start)
// residual after the pre-smoothing sweep z1 = omega D^-1 r: r1 = r - S z1 at
// node i (pin 0)
__device__ __forceinline__ double pre_residual(const LGrid& g, const double* r, double omega, int i, int i0, int i1) {
  auto zf = [&](int j) -> double { return (j == g.pin) ? 0.0 : omega * g.dinvS[j] * r[j]; };
  double v = 0.0;
  if (i != g.pin) {
    const double sm0 = (i0 > 0) ? g.s0[i - g.n1] : 0.0, sp0 = g.s0[i];
    const double sm1 = (i1 > 0) ? g.s1[i - 1] : 0.0, sp1 = g.s1[i];
    double off = 0.0;
    if (i0 > 0) off += sm0 * zf(i - g.n1);
    if (i0 < g.n0 - 1) off += sp0 * zf(i + g.n1);
    if (i1 > 0) off += sm1 * zf(i - 1);
    if (i1 < g.n1 - 1) off += sp1 * zf(i + 1);
    v = r[i] - ((sm0 + sp0 + sm1 + sp1) * zf(i) - off);
  }
  return v;
}

__global__ void vc_pre_kernel(LGrid g, const double* r, double omega, const FcgState* st, double* r1) {
  tpf::chain_begin();
  if (st && st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    r1[i] = pre_residual(g, r, omega, i, i0, i1);
  }
  tpf::chain_end();
}

// rc = R r1 (block sums); partials of rc^2 / D_c
__global__ void __launch_bounds__(kRedThreads) restrict_kernel(LGrid g, const double* r1, double* rc,
                                                               const FcgState* st, double* part) {
  tpf::chain_begin();
  double v[1] = {0.0};
  if (!(st && st->done)) {
    const int nc = g.nc0 * g.nc1;
    for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
      const int I0 = I / g.nc1, I1 = I - I0 * g.nc1;
      double acc = 0.0;
      for (int a0 = I0 * g.b; a0 < min(g.n0, (I0 + 1) * g.b); ++a0)
        for (int a1 = I1 * g.b; a1 < min(g.n1, (I1 + 1) * g.b); ++a1) acc += r1[a0 * g.n1 + a1];
      rc[I] = acc;
      const double q = acc * g.dcis[I];
      v[0] += q * q;
    }
  }
  block_partials<1>(v, part);
  tpf::chain_end();
}

// pre-smoothing, restriction and the coarse input scale in one launch:
// rc = R r1 with each fine node's pre-smoothed residual r1 formed once on the
// fly (the vc_pre_kernel formula), b lanes per aggregate adding its rows by a
// shuffle tree, partials of (rc D_c^-1/2)^2; the last block to finish sums
// the partials in block order into the input scale s_c and, inside the
// flexible GMRES cycle (gdone non-null), copies the cycle's done flag into
// st->done for the kernels after it
__global__ void __launch_bounds__(kRedThreads) restrict_pre_kernel(LGrid g, const double* r, double omega,
                                                                   FcgState* st, const int* gdone, double* rc,
                                                                   double* part, unsigned* arrive) {
  tpf::chain_begin();
  const bool skip = gdone ? (*gdone != 0) : (st->done != 0);
  const int nc = g.nc0 * g.nc1;
  double v[1] = {0.0};
  if (!skip) {
    // b consecutive lanes per aggregate (b = 2, 4 or 8 divides the warp), lane
    // k summing fine row k of the aggregate; the row sums are added by a
    // shuffle tree.  Whole warps iterate together (the shuffles need every lane).
    const int b = g.b;
    const long long total = (long long)nc * b;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t0 = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); t0 < total; t0 += stride) {
      const long long t = t0 + (threadIdx.x & 31);
      const bool on = t < total;
      const int I = on ? (int)(t / b) : 0, k = on ? (int)(t - (long long)I * b) : 0;
      const int I0 = I / g.nc1, I1 = I - I0 * g.nc1;
      const int a0 = I0 * b + k;
      double acc = 0.0;
      if (on && a0 < g.n0)
        for (int a1 = I1 * b; a1 < min(g.n1, (I1 + 1) * b); ++a1)
          acc += pre_residual(g, r, omega, a0 * g.n1 + a1, a0, a1);
      for (int off = b >> 1; off >= 1; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (on && k == 0) {
        rc[I] = acc;
        const double q = acc * g.dcis[I];
        v[0] += q * q;
      }
    }
  }
  block_partials<1>(v, part);
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (s_last) {
    __threadfence();
    double t[1];
    reduce_partials<1>(part, gridDim.x, t);
    if (threadIdx.x == 0) {
      if (!skip) {
        const double sc = sqrt(t[0] / nc);
        st->sc = sc;
        st->inv_sc = sc > 0.0 ? 1.0 / sc : 0.0;
      }
      if (gdone) st->done = *gdone;
      *arrive = 0u;
    }
  }
  tpf::chain_end();
}

// scaled Galerkin couplings of aggregate I to the next row / column
__device__ __forceinline__ void coarse_coupl(const LGrid& g, const double* cc0, const double* cc1, int I, int y,
                                             int x, float& a0, float& a1) {
  a0 = (y + 1 < g.nc0) ? (float)(cc0[I] * g.dcis[I] * g.dcis[I + g.nc1]) : 0.f;
  a1 = (x + 1 < g.nc1) ? (float)(cc1[I] * g.dcis[I] * g.dcis[I + 1]) : 0.f;
}

// network input on the coarse image: (D_c^-1/2 rc / s_c, c~_c, coarse couplings)
__global__ void pack_coarse_kernel(LGrid g, const double* rc, const double* cc0, const double* cc1,
                                   const FcgState* st, bf16* xin) {
  tpf::chain_begin();
  tpf::tc::pdl_trigger();
  if (st->done) return;
  const int Wp = g.W + 2;
  const long long P = (long long)(g.H + 2) * Wp;
  const double inv = st->inv_sc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x) {
    const int yy = (int)(q / Wp), xx = (int)(q - (long long)yy * Wp);
    const int y = yy - 1, x = xx - 1;
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
    if (y >= 0 && y < g.nc0 && x >= 0 && x < g.nc1) {
      const int I = y * g.nc1 + x;
      c0 = (float)(rc[I] * g.dcis[I] * inv);
      c1 = g.featc[I];
      coarse_coupl(g, cc0, cc1, I, y, x, c2, c3);
    }
    uint4* o = reinterpret_cast<uint4*>(xin + q * 16);
    o[0] = pack4bf(c0, c1, c2, c3);
    o[1] = make_uint4(0, 0, 0, 0);
  }
  tpf::chain_end();
}

// z2 = w D^-1 r + P (s_c D_c^-1/2 y), pin 0
__global__ void prolong_kernel(LGrid g, const float* y, const double* r, double omega, const FcgState* st,
                               double* z2) {
  tpf::chain_begin();
  if (st->done) return;
  const double sc = st->sc;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    z2[i] = prolong_value(g, y, r, omega, sc, i, i0, i1);
  }
  tpf::chain_end();
}

// prolongation fused with the first post-smoothing sweep:
// z2 = w D^-1 r + P (s_c D_c^-1/2 y) evaluated on the fly at the node and its
// neighbours, z = z2 + w D^-1 (r - S z2), pin 0
__global__ void prolong_smooth_kernel(LGrid g, const float* y, const double* r, double omega, const FcgState* st,
                                      double* z) {
  tpf::chain_begin();
  if (st->done) return;
  const double sc = st->sc;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    if (i == g.pin) {
      z[i] = 0.0;
      continue;
    }
    const bool h0m = i0 > 0, h0p = i0 < g.n0 - 1, h1m = i1 > 0, h1p = i1 < g.n1 - 1;
    z[i] = jacobi_node(prolong_value(g, y, r, omega, sc, i, i0, i1),
                       h0m ? prolong_value(g, y, r, omega, sc, i - g.n1, i0 - 1, i1) : 0.0,
                       h0p ? prolong_value(g, y, r, omega, sc, i + g.n1, i0 + 1, i1) : 0.0,
                       h1m ? prolong_value(g, y, r, omega, sc, i - 1, i0, i1 - 1) : 0.0,
                       h1p ? prolong_value(g, y, r, omega, sc, i + 1, i0, i1 + 1) : 0.0,
                       h0m ? g.s0[i - g.n1] : 0.0, g.s0[i], h1m ? g.s1[i - 1] : 0.0, g.s1[i], h0m, h0p, h1m, h1p,
                       g.dinvS[i], r[i], omega);
  }
  tpf::chain_end();
}

// training pair of the coarse problem: e1 = e - w D^-1 r (error after the
// pre-smoothing sweep), target = D_c^1/2 mean_I(e1) / s_c on the coarse image
__global__ void pair_coarse_write_kernel(LGrid g, const double* e, const double* r, const double* rc,
                                         const double* cc0, const double* cc1, double omega, const double* part,
                                         int nb, float* in, float* target) {
  __shared__ double s_inv;
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int i = 0; i < nb; ++i) a += part[i];
    const double sc = sqrt(a / (g.nc0 * g.nc1));
    s_inv = (sc > 0.0) ? 1.0 / sc : 0.0;
  }
  __syncthreads();
  const double inv = s_inv;
  const long long n = (long long)g.H * g.W;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(q / g.W), x = (int)(q - (long long)y * g.W);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, t = 0.f;
    if (y < g.nc0 && x < g.nc1) {
      const int I = y * g.nc1 + x;
      double acc = 0.0;
      int cnt = 0;
      for (int i0 = y * g.b; i0 < min(g.n0, (y + 1) * g.b); ++i0)
        for (int i1 = x * g.b; i1 < min(g.n1, (x + 1) * g.b); ++i1) {
          const int i = i0 * g.n1 + i1;
          acc += (i == g.pin) ? 0.0 : e[i] - omega * g.dinvS[i] * r[i];
          ++cnt;
        }
      const double d = g.dcis[I];
      a0 = (float)(rc[I] * d * inv);
      a1 = g.featc[I];
      coarse_coupl(g, cc0, cc1, I, y, x, a2, a3);
      t = (d > 0.0) ? (float)((acc / cnt) / d * inv) : 0.f;
    }
    in[4 * q] = a0;
    in[4 * q + 1] = a1;
    in[4 * q + 2] = a2;
    in[4 * q + 3] = a3;
    target[q] = t;
  }
}

// energy-loss data of a coarse training pair: scaled Galerkin couplings of the
// coarse operator on the network image (coupl[q][0]: to the next row,
// coupl[q][1]: to the next column; A~ = D_c^-1/2 A_c D_c^-1/2 = I - couplings)
// and E~ = (e1 . S e1) / s_c^2 = (e1 . r1) / s_c^2
__global__ void coarse_coupl_write_kernel(LGrid g, const double* c0, const double* c1, float* coupl) {
  const long long n = (long long)g.H * g.W;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(q / g.W), x = (int)(q - (long long)y * g.W);
    float a = 0.f, b = 0.f;
    if (y < g.nc0 && x < g.nc1) {
      const int I = y * g.nc1 + x;
      if (y + 1 < g.nc0) a = (float)(c0[I] * g.dcis[I] * g.dcis[I + g.nc1]);
      if (x + 1 < g.nc1) b = (float)(c1[I] * g.dcis[I] * g.dcis[I + 1]);
    }
    coupl[2 * q] = a;
    coupl[2 * q + 1] = b;
  }
}

// partial sums of e1 . r1 with e1 = e - w D^-1 r (pin 0)
__global__ void __launch_bounds__(kRedThreads) energy_partials_kernel(LGrid g, const double* e, const double* r,
                                                                      const double* r1, double omega, double* part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    if (i == g.pin) continue;
    v[0] += (e[i] - omega * g.dinvS[i] * r[i]) * r1[i];
  }
  block_partials<1>(v, part);
}

// E~ = (e1 . r1) / s_c^2, s_c from the restriction partials
__global__ void energy_scale_kernel(LGrid g, const double* part_e, const double* part_r, int nb, double* escale) {
  double v[1], w[1];
  reduce_partials<1>(part_e, nb, v);
  reduce_partials<1>(part_r, nb, w);
  if (threadIdx.x == 0) {
    const double sc2 = w[0] / (g.nc0 * g.nc1);
    escale[0] = (sc2 > 0.0) ? v[0] / sc2 : 1.0;
  }
}

inline int ew_blocks(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 8)); }

}  // namespace

struct tpf_lppe {
  tpf_ppe* ppe = nullptr;
  tpf_unet* net = nullptr;
  tpf::PpeView v{};
  LGrid g{};
  double *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *z2 = nullptr, *w = nullptr, *pp = nullptr,
         *qp = nullptr, *part = nullptr;   // pp / qp: kMaxWin stored directions P_j, S P_j
  float* feat = nullptr;
  unsigned long long* rmax = nullptr;
  // two-level mode
  double *r1 = nullptr, *rc = nullptr, *dc = nullptr, *dcis = nullptr, *cc0 = nullptr, *cc1 = nullptr,
         *part2 = nullptr;
  float* featc = nullptr;
  double graph_pre_omega = 0.0;
  FcgState* st = nullptr;
  FcgState* st_host = nullptr;   // pinned
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_smooth = -1;
  double graph_omega = 0.0;
  int win = 1;            // window of the current solve
  int graph_win = -1;
  bool have_feat = false;
  // flexible GMRES outer method: bases V (restart + 1) and Z (restart), the
  // Hessenberg block, partials, state, residual / operator scratch, graph
  int gm_cap = 0;
  double *gV = nullptr, *gZ = nullptr, *ggm = nullptr, *gpart = nullptr, *gr = nullptr, *gw = nullptr,
         *gt = nullptr;
  int gpart_len = 0;
  GmState* ggst = nullptr;
  cudaGraphExec_t gexec = nullptr;
  long long gkey[6] = {0, 0, 0, 0, 0, 0};
  int smooth_block = 4;   // sweeps per smoother launch (1: one sweep per launch)
  unsigned* arrive = nullptr;   // last-block counter of restrict_pre_kernel (zero between launches)
  std::vector<void*> allocs;
};

namespace {

template <typename T>
int lalloc(tpf_lppe* lp, T** p, size_t n) {
  if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    tpf::set_error("cudaMalloc of %zu bytes failed", n * sizeof(T));
    return TPF_ECUDA;
  }
  lp->allocs.push_back(*p);
  return TPF_OK;
}

int refresh_view(tpf_lppe* lp) {
  int st = tpf::ppe_view(lp->ppe, &lp->v);
  if (st) return st;
  lp->g.s0 = lp->v.s[0];
  lp->g.s1 = lp->v.s[1];
  lp->g.dinvS = lp->v.dinvS;
  lp->g.dv0 = lp->v.dv[0];
  lp->g.dv1 = lp->v.dv[1];
  return TPF_OK;
}

int features(tpf_lppe* lp, const double* rho, cudaStream_t s) {
  TPF_CUDA_TRY(cudaMemsetAsync(lp->rmax, 0, sizeof(unsigned long long), s));
  rho_max_kernel<<<ew_blocks(lp->g.ndof), 256, 0, s>>>(lp->g.ndof, rho, lp->rmax);
  feature_kernel<<<ew_blocks(lp->g.ndof), 256, 0, s>>>(lp->g.ndof, rho, lp->rmax, lp->feat);
  if (lp->g.b > 1) {
    const int nc = lp->g.nc0 * lp->g.nc1;
    coarse_operator_kernel<<<ew_blocks(nc), 256, 0, s>>>(lp->g, lp->dc, lp->cc0, lp->cc1);
    coarse_setup_kernel<<<ew_blocks(nc), 256, 0, s>>>(lp->g, lp->dc, lp->feat, lp->dcis, lp->featc);
  }
  TPF_CUDA_TRY(cudaGetLastError());
  lp->have_feat = true;
  return TPF_OK;
}

// z = B(r): network (+ smoothing); result in lp->z (smooth even) or lp->z2
// n damped-Jacobi sweeps ping-ponging between cur and other (cur ends holding
// the result): smooth_block sweeps per launch
// (the residual is rin; with last_out non-null the final launch writes there
// and cur ends as last_out)
void enqueue_sweeps(tpf_lppe* lp, int n, double omega, cudaStream_t s, const double* rin, double*& cur,
                    double*& other, double* last_out = nullptr) {
  const LGrid& g = lp->g;
  if (lp->smooth_block <= 1) {
    for (int k = 0; k < n; ++k) {
      double* dst = (last_out && k == n - 1) ? last_out : other;
      tpf::launch_chained(fcg_smooth_kernel, ew_blocks(g.ndof), 256, 0, s, g, cur, rin, omega, lp->st, dst);
      other = cur;
      cur = dst;
    }
    return;
  }
  const int tiles = ((g.n0 + kSmTY - 1) / kSmTY) * ((g.n1 + kSmTX - 1) / kSmTX);
  for (int k = 0; k < n; k += lp->smooth_block) {
    const int kk = std::min(lp->smooth_block, n - k);
    double* dst = (last_out && k + kk >= n) ? last_out : other;
    tpf::launch_chained(smooth_block_kernel, tiles, kSmThreads, 0, s, g, cur, static_cast<const float*>(nullptr), rin,
                        omega, kk, lp->st, dst);
    other = cur;
    cur = dst;
  }
}

// z = B(r).  Two-level mode: rin (default lp->r) is read in place; with zfinal
// non-null the last kernel writes z there; gdone: the flexible GMRES cycle's
// done flag (the preconditioner's kernels skip once it is set).
int enqueue_precond(tpf_lppe* lp, int smooth, double omega, cudaStream_t s, double** zout,
                    const double* rin = nullptr, double* zfinal = nullptr, const int* gdone = nullptr) {
  const LGrid& g = lp->g;
  if (g.b > 1) {
    if (!rin) rin = lp->r;
    tpf::launch_chained(restrict_pre_kernel, kRedBlocks, kRedThreads, 0, s, g, rin, omega, lp->st, gdone, lp->rc,
                        lp->part, lp->arrive);
    tpf::launch_chained(pack_coarse_kernel, ew_blocks((g.H + 2) * (g.W + 2)), 256, 0, s, g, lp->rc, lp->cc0,
                        lp->cc1, lp->st, tpf::unet_input(lp->net));
    TPF_CUDA_TRY(cudaGetLastError());
    int st = tpf::unet_forward_packed(lp->net, 1, s);
    if (st) return st;
    // the prolongation sweep and the next ones: with the blocked smoother the
    // first launch starts from the prolongated correction itself
    const int first_sweeps = (smooth > 0 && lp->smooth_block > 1) ? std::min(smooth, lp->smooth_block)
                                                                   : std::min(smooth, 1);
    double* first = (zfinal && smooth <= first_sweeps) ? zfinal : lp->z;
    if (first_sweeps > 1) {
      const int tiles = ((g.n0 + kSmTY - 1) / kSmTY) * ((g.n1 + kSmTX - 1) / kSmTX);
      tpf::launch_chained(smooth_block_kernel, tiles, kSmThreads, 0, s, g, static_cast<const double*>(nullptr),
                          static_cast<const float*>(tpf::unet_output(lp->net)), rin, omega, first_sweeps, lp->st,
                          first);
    } else if (smooth > 0) {
      tpf::launch_chained(prolong_smooth_kernel, ew_blocks(g.ndof), 256, 0, s, g, tpf::unet_output(lp->net), rin,
                          omega, lp->st, first);
    } else {
      tpf::launch_chained(prolong_kernel, ew_blocks(g.ndof), 256, 0, s, g, tpf::unet_output(lp->net), rin, omega,
                          lp->st, first);
    }
    double* cur = first;
    double* other = lp->z2;
    enqueue_sweeps(lp, smooth - first_sweeps, omega, s, rin, cur, other, zfinal);
    TPF_CUDA_TRY(cudaGetLastError());
    *zout = cur;
    return TPF_OK;
  }
  tpf::launch_chained(fcg_pack_kernel, ew_blocks((g.H + 2) * (g.W + 2)), 256, 0, s, g, lp->r, lp->feat, lp->st,
                      tpf::unet_input(lp->net));
  TPF_CUDA_TRY(cudaGetLastError());
  int st = tpf::unet_forward_packed(lp->net, 1, s);
  if (st) return st;
  tpf::launch_chained(fcg_unpack_kernel, ew_blocks(g.ndof), 256, 0, s, g, tpf::unet_output(lp->net), lp->st, lp->z);
  double* cur = lp->z;
  double* other = lp->z2;
  enqueue_sweeps(lp, smooth, omega, s, lp->r, cur, other);
  TPF_CUDA_TRY(cudaGetLastError());
  *zout = cur;
  return TPF_OK;
}

// ---- flexible GMRES outer method (fgmres_solve, gmres.cuh) ------------------------------

// the preconditioner's input v (a basis vector) into r, with the partials of
// its D^-1-weighted norm (the network input scale); nothing once the cycle is done
__global__ void __launch_bounds__(kRedThreads) fgm_in_kernel(LGrid g, const double* v, const int* gdone, double* r,
                                                             double* part) {
  tpf::chain_begin();
  double acc[1] = {0.0};
  if (!*gdone) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
      const double vi = v[i];
      r[i] = vi;
      acc[0] += vi * vi * g.dinvS[i];
    }
  }
  block_partials<1>(acc, part);
  tpf::chain_end();
}

// the scale s of the network input and the preconditioner kernels' skip flag
__global__ void fgm_scale_kernel(const double* part, int nb, int ndof, const int* gdone, FcgState* st) {
  tpf::chain_begin();
  double v[1];
  reduce_partials<1>(part, nb, v);
  if (threadIdx.x == 0) {
    st->done = *gdone;
    set_scale(st, v[0], ndof);
  }
  tpf::chain_end();
}

__global__ void fgm_out_kernel(int n, const double* z, const int* gdone, double* out) {
  tpf::chain_begin();
  if (*gdone) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = z[i];
  tpf::chain_end();
}

// w = S z with the pinned row w[pin] = z[pin] (z[pin] = 0 on this Krylov space)
__global__ void fgm_apply_kernel(LGrid g, const double* z, const int* gdone, double* w) {
  tpf::chain_begin();
  if (gdone && *gdone) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.ndof; i += gridDim.x * blockDim.x) {
    const int i0 = i / g.n1, i1 = i - i0 * g.n1;
    w[i] = (i == g.pin) ? z[i] : s_apply(g, z, i, i0, i1);
  }
  tpf::chain_end();
}

// one flexible-CG step with M stored directions (the window length picks the instance)
template <int M>
void enqueue_fcg_step(tpf_lppe* lp, const double* z, cudaStream_t s) {
  const LGrid& g = lp->g;
  fcg_sdot_kernel<M><<<kRedBlocks, kRedThreads, 0, s>>>(g, z, lp->r, lp->pp, lp->qp, lp->w, lp->st, lp->part);
  fcg_coef_kernel<M><<<1, 256, 0, s>>>(lp->part, kRedBlocks, lp->st);
  fcg_update_kernel<M><<<kRedBlocks, kRedThreads, 0, s>>>(g, z, lp->w, lp->pp, lp->qp, lp->x, lp->r, lp->st,
                                                          lp->part);
}

int enqueue_iteration(tpf_lppe* lp, int smooth, double omega, cudaStream_t s) {
  double* z = nullptr;
  int st = enqueue_precond(lp, smooth, omega, s, &z);
  if (st) return st;
  const LGrid& g = lp->g;
  if (lp->win <= 1) {
    enqueue_fcg_step<1>(lp, z, s);
  } else if (lp->win <= 2) {
    enqueue_fcg_step<2>(lp, z, s);
  } else if (lp->win <= 4) {
    enqueue_fcg_step<4>(lp, z, s);
  } else {
    enqueue_fcg_step<kMaxWin>(lp, z, s);
  }
  fcg_finish_iter_kernel<<<1, 256, 0, s>>>(lp->part, kRedBlocks, g.ndof, lp->st);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int build_graph(tpf_lppe* lp, int smooth, double omega) {
  if (lp->exec && lp->graph_smooth == smooth && lp->graph_omega == omega && lp->graph_win == lp->win) return TPF_OK;
  if (lp->exec) {
    cudaGraphExecDestroy(lp->exec);
    lp->exec = nullptr;
  }
  cudaGraph_t graph = nullptr;
  TPF_CUDA_TRY(cudaStreamBeginCapture(lp->cap, cudaStreamCaptureModeThreadLocal));
  int st = enqueue_iteration(lp, smooth, omega, lp->cap);
  cudaError_t e = cudaStreamEndCapture(lp->cap, &graph);
  if (st) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) {
    tpf::set_error("graph capture of the FCG iteration failed: %s", cudaGetErrorString(e));
    return TPF_ECUDA;
  }
  e = cudaGraphInstantiate(&lp->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    lp->exec = nullptr;
    tpf::set_error("graph instantiation failed: %s", cudaGetErrorString(e));
    return TPF_ECUDA;
  }
  lp->graph_smooth = smooth;
  lp->graph_omega = omega;
  lp->graph_win = lp->win;
  return TPF_OK;
}

// flexible GMRES workspace for restart length R (kept for the handle's life)
int ensure_fgmres_work(tpf_lppe* lp, int R) {
  if (lp->gm_cap >= R) return TPF_OK;
  const int n = lp->g.ndof;
  int st;
  const size_t gm_len = (size_t)R * (R + 2) + 2 * (size_t)R + (size_t)(R + 1) * 4 + 8;
  const int part_len = (R + 2) * std::max(1, 4 * tpf::sm_count());
  if ((st = lalloc(lp, &lp->gV, (size_t)(R + 1) * n)) || (st = lalloc(lp, &lp->gZ, (size_t)R * n)) ||
      (st = lalloc(lp, &lp->ggm, gm_len)) || (st = lalloc(lp, &lp->gpart, (size_t)part_len)) ||
      (st = lalloc(lp, &lp->gr, (size_t)n)) || (st = lalloc(lp, &lp->gw, (size_t)n)) ||
      (st = lalloc(lp, &lp->gt, (size_t)n)) || (st = lalloc(lp, &lp->ggst, 1)))
    return st;
  if (lp->gexec) {
    cudaGraphExecDestroy(lp->gexec);
    lp->gexec = nullptr;
  }
  lp->gpart_len = part_len;
  lp->gm_cap = R;
  return TPF_OK;
}

// the learned solve with flexible GMRES(R) as the outer method: the same
// weighted system and network application as the flexible CG, each basis
// vector preconditioned by the network (its own input scale), x += Z y per
// cycle; returns whether the true residual met the tolerance
int solve_fgmres(tpf_lppe* lp, const tpf_learned_options& o, cudaStream_t s, bool x_nonzero, GmresOutcome& out) {
  const LGrid& g = lp->g;
  int st;
  if ((st = ensure_fgmres_work(lp, o.restart))) return st;
  GmresWork W;
  W.n = g.ndof;
  W.ew_blocks = ew_blocks(g.ndof);
  W.part_len = lp->gpart_len;
  W.restart_cap = lp->gm_cap;
  W.V = lp->gV;
  W.gm = lp->ggm;
  W.part = lp->gpart;
  W.gst = lp->ggst;
  W.b = lp->b;
  W.x = lp->x;
  W.r = lp->gr;
  W.w = lp->gw;
  W.t = lp->gt;
  W.exec = &lp->gexec;
  W.cap = &lp->cap;
  W.key = lp->gkey;
  auto apply = [&](const double* in, double* outv, cudaStream_t cs, const int* done) -> int {
    tpf::launch_chained(fgm_apply_kernel, ew_blocks(g.ndof), 256, 0, cs, g, in, done, outv);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  };
  auto resid = [&](const double* x, double* r, cudaStream_t cs) -> int {
    fcg_residual_kernel<<<kRedBlocks, kRedThreads, 0, cs>>>(g, lp->b, x, r, lp->part);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  };
  auto precond = [&](const double* in, double* outv, cudaStream_t cs, const int* done) -> int {
    if (g.b > 1) {
      // the basis vector is read in place and z lands in the Z column; the
      // two-level path needs no fine-grid input scale
      double* z = nullptr;
      return enqueue_precond(lp, o.smooth, o.omega, cs, &z, in, outv, done);
    }
    tpf::launch_chained(fgm_in_kernel, kRedBlocks, kRedThreads, 0, cs, g, in, done, lp->r, lp->part);
    tpf::launch_chained(fgm_scale_kernel, 1, 256, 0, cs, lp->part, kRedBlocks, g.ndof, done, lp->st);
    double* z = nullptr;
    int est = enqueue_precond(lp, o.smooth, o.omega, cs, &z);
    if (est) return est;
    tpf::launch_chained(fgm_out_kernel, ew_blocks(g.ndof), 256, 0, cs, g.ndof, z, done, outv);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  };
  const long long cycles = std::max<long long>(1, (o.maxiter + o.restart - 1) / o.restart);
  const long long key_a = (long long)o.smooth * 1000003LL + (long long)(o.omega * 1e9);
  // the flexible CG's stall rule, checked after each cycle on the true residual
  const long long stall_iters =
      (o.fallback && o.stall_checks > 0) ? (long long)o.stall_checks * o.check_every : 0;
  return fgmres_solve(W, lp->gZ, o.restart, o.tol, cycles, x_nonzero, key_a, (long long)(intptr_t)lp->st, apply,
                      resid, precond, s, out, o.stall_factor, stall_iters);
}

int read_state(tpf_lppe* lp, cudaStream_t s) {
  TPF_CUDA_TRY(cudaMemcpyAsync(lp->st_host, lp->st, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  return tpf::unet_check(lp->net, s);
}

int true_residual(tpf_lppe* lp, cudaStream_t s, double tol, int first, int win) {
  fcg_residual_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(lp->g, lp->b, lp->x, lp->r, lp->part);
  fcg_start_kernel<<<1, 256, 0, s>>>(lp->part, kRedBlocks, lp->g.ndof, lp->st, tol, first, win);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

}  // namespace

extern "C" {

void tpf_lppe_default_options(tpf_learned_options* o) {
  if (!o) return;
  o->tol = 1e-8;
  o->maxiter = 2000;
  o->smooth = 16;
  o->omega = 0.8;
  o->check_every = 8;
  o->stall_checks = 16;
  o->stall_factor = 0.5;
  o->fallback = 1;
  o->use_graph = 1;
  o->window = 8;
  o->outer = 1;
  o->restart = 60;
}

int tpf_lppe_create(tpf_lppe** out, tpf_ppe* ppe, tpf_unet* net, int coarsen) {
  TPF_CHECK_ARG(out && ppe && net, "NULL argument");
  TPF_CHECK_ARG(coarsen == 1 || coarsen == 2 || coarsen == 4 || coarsen == 8, "coarsen must be 1, 2, 4 or 8");
  auto* lp = new tpf_lppe();
  lp->ppe = ppe;
  lp->net = net;
  auto fail = [&](int code) {
    for (void* p : lp->allocs) cudaFree(p);
    if (lp->st_host) cudaFreeHost(lp->st_host);
    if (lp->cap) cudaStreamDestroy(lp->cap);
    delete lp;
    return code;
  };
  int st = tpf::ppe_view(ppe, &lp->v);
  if (st) return fail(st);
  if (lp->v.ndim != 2) {
    tpf::set_error("the learned preconditioner is two-dimensional (got ndim=%d)", lp->v.ndim);
    return fail(TPF_EINVAL);
  }
  int H = 0, W = 0, mb = 0;
  tpf::unet_dims(net, &H, &W, &mb);
  const int nc0 = (lp->v.n0 + coarsen - 1) / coarsen, nc1 = (lp->v.n1 + coarsen - 1) / coarsen;
  const int Hn = (nc0 + 7) / 8 * 8, Wn = (nc1 + 7) / 8 * 8;
  if (H != Hn || W != Wn) {
    tpf::set_error("U-Net image %dx%d does not match the grid: need %dx%d (%s rounded up to 8)", H, W, Hn, Wn,
                   coarsen > 1 ? "aggregates" : "nodes");
    return fail(TPF_EINVAL);
  }
  lp->g.b = coarsen;
  lp->g.nc0 = nc0;
  lp->g.nc1 = nc1;
  lp->g.n0 = lp->v.n0;
  lp->g.n1 = lp->v.n1;
  lp->g.ndof = lp->v.ndof;
  lp->g.pin = lp->v.pin;
  lp->g.H = H;
  lp->g.W = W;
  const size_t n = lp->v.ndof;
  if ((st = lalloc(lp, &lp->b, n)) || (st = lalloc(lp, &lp->x, n)) || (st = lalloc(lp, &lp->r, n)) ||
      (st = lalloc(lp, &lp->z, n)) || (st = lalloc(lp, &lp->z2, n)) || (st = lalloc(lp, &lp->w, n)) ||
      (st = lalloc(lp, &lp->pp, kMaxWin * n)) || (st = lalloc(lp, &lp->qp, kMaxWin * n)) ||
      (st = lalloc(lp, &lp->part, (2 * kMaxWin + 4) * kRedBlocks)) ||
      (st = lalloc(lp, &lp->feat, n)) || (st = lalloc(lp, &lp->rmax, 1)) || (st = lalloc(lp, &lp->st, 1)))
    return fail(st);
  if (coarsen > 1) {
    const size_t nc = (size_t)nc0 * nc1;
    if ((st = lalloc(lp, &lp->r1, n)) || (st = lalloc(lp, &lp->rc, nc)) || (st = lalloc(lp, &lp->dc, nc)) ||
        (st = lalloc(lp, &lp->dcis, nc)) || (st = lalloc(lp, &lp->featc, nc)) || (st = lalloc(lp, &lp->cc0, nc)) ||
        (st = lalloc(lp, &lp->cc1, nc)) || (st = lalloc(lp, &lp->part2, kRedBlocks)) ||
        (st = lalloc(lp, &lp->arrive, 1)))
      return fail(st);
    if (cudaMemset(lp->arrive, 0, sizeof(unsigned)) != cudaSuccess) {
      cudaGetLastError();
      tpf::set_error("cudaMemset failed");
      return fail(TPF_ECUDA);
    }
    lp->g.dcis = lp->dcis;
    lp->g.featc = lp->featc;
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&lp->st_host), sizeof(FcgState)) != cudaSuccess) {
    cudaGetLastError();
    lp->st_host = nullptr;
    tpf::set_error("cudaMallocHost failed");
    return fail(TPF_ECUDA);
  }
  if (cudaStreamCreateWithFlags(&lp->cap, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    lp->cap = nullptr;
    tpf::set_error("cudaStreamCreate failed");
    return fail(TPF_ECUDA);
  }
  *out = lp;
  return TPF_OK;
}

int tpf_lppe_destroy(tpf_lppe* lp) {
  if (!lp) return TPF_OK;
  cudaDeviceSynchronize();
  if (lp->exec) cudaGraphExecDestroy(lp->exec);
  if (lp->gexec) cudaGraphExecDestroy(lp->gexec);
  for (void* p : lp->allocs) cudaFree(p);
  if (lp->st_host) cudaFreeHost(lp->st_host);
  if (lp->cap) cudaStreamDestroy(lp->cap);
  delete lp;
  return TPF_OK;
}

int tpf_lppe_prepare(tpf_lppe* lp, const double* rho, void* stream) {
  TPF_CHECK_ARG(lp && rho, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = tpf_ppe_prepare(lp->ppe, rho, stream);
  if (st) return st;
  if ((st = refresh_view(lp))) return st;
  return features(lp, rho, s);
}

int tpf_lppe_pair(tpf_lppe* lp, const double* e, float* in2, float* target, double omega, void* stream) {
  TPF_CHECK_ARG(lp && e && in2 && target, "NULL argument");
  TPF_CHECK_ARG(lp->have_feat, "call tpf_lppe_prepare first");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (lp->g.b > 1) {
    pair_residual_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(lp->g, e, lp->r, lp->part);
    tpf::launch_chained(vc_pre_kernel, ew_blocks(lp->g.ndof), 256, 0, s, lp->g, lp->r, omega, nullptr, lp->r1);
    tpf::launch_chained(restrict_kernel, kRedBlocks, kRedThreads, 0, s, lp->g, lp->r1, lp->rc, nullptr, lp->part);
    pair_coarse_write_kernel<<<ew_blocks(lp->g.H * lp->g.W), 256, 0, s>>>(lp->g, e, lp->r, lp->rc, lp->cc0, lp->cc1,
                                                                         omega, lp->part, kRedBlocks, in2, target);
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  }
  pair_residual_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(lp->g, e, lp->r, lp->part);
  pair_write_kernel<<<ew_blocks(lp->g.H * lp->g.W), 256, 0, s>>>(lp->g, e, lp->r, lp->feat, lp->part, kRedBlocks,
                                                                 in2, target);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int tpf_lppe_pair_energy(tpf_lppe* lp, const double* e, float* in2, float* coupl, double* escale, double omega,
                         void* stream) {
  TPF_CHECK_ARG(lp && e && in2 && coupl && escale, "NULL argument");
  TPF_CHECK_ARG(lp->have_feat, "call tpf_lppe_prepare first");
  TPF_CHECK_ARG(lp->g.b > 1, "energy pairs need the two-level mode (coarsen > 1)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LGrid& g = lp->g;
  pair_residual_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(g, e, lp->r, lp->part);
  tpf::launch_chained(vc_pre_kernel, ew_blocks(g.ndof), 256, 0, s, g, lp->r, omega, nullptr, lp->r1);
  tpf::launch_chained(restrict_kernel, kRedBlocks, kRedThreads, 0, s, g, lp->r1, lp->rc, nullptr, lp->part);
  // in2 (channel 0 = scaled restricted residual, channel 1 = feature); the target is unused
  pair_coarse_write_kernel<<<ew_blocks(g.H * g.W), 256, 0, s>>>(g, e, lp->r, lp->rc, lp->cc0, lp->cc1, omega,
                                                                lp->part, kRedBlocks, in2,
                                                                reinterpret_cast<float*>(lp->z2));
  energy_partials_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(g, e, lp->r, lp->r1, omega, lp->part2);
  energy_scale_kernel<<<1, 256, 0, s>>>(g, lp->part2, lp->part, kRedBlocks, escale);
  coarse_coupl_write_kernel<<<ew_blocks(g.H * g.W), 256, 0, s>>>(g, lp->cc0, lp->cc1, coupl);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int tpf_lppe_set_smooth_block(tpf_lppe* lp, int sweeps) {
  TPF_CHECK_ARG(lp, "NULL argument");
  TPF_CHECK_ARG(sweeps >= 1 && sweeps <= kSmK, "sweeps per smoother launch must be in [1, 4]");
  if (sweeps != lp->smooth_block) {
    // the captured iteration / cycle graphs hold the old launches
    if (lp->exec) { cudaGraphExecDestroy(lp->exec); lp->exec = nullptr; }
    if (lp->gexec) { cudaGraphExecDestroy(lp->gexec); lp->gexec = nullptr; }
    lp->graph_smooth = -1;
    lp->smooth_block = sweeps;
  }
  return TPF_OK;
}

int tpf_lppe_smooth(tpf_lppe* lp, const double* zin, const double* r, double* zout, int sweeps, double omega,
                    void* stream) {
  TPF_CHECK_ARG(lp && zin && r && zout, "NULL argument");
  TPF_CHECK_ARG(lp->have_feat, "call tpf_lppe_prepare first");
  TPF_CHECK_ARG(sweeps >= 0 && sweeps <= 1024, "sweeps must be in [0, 1024]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = sizeof(double) * lp->g.ndof;
  TPF_CUDA_TRY(cudaMemsetAsync(&lp->st->done, 0, sizeof(int), s));
  TPF_CUDA_TRY(cudaMemcpyAsync(lp->r, r, bytes, cudaMemcpyDeviceToDevice, s));
  TPF_CUDA_TRY(cudaMemcpyAsync(lp->z, zin, bytes, cudaMemcpyDeviceToDevice, s));
  double* cur = lp->z;
  double* other = lp->z2;
  enqueue_sweeps(lp, sweeps, omega, s, lp->r, cur, other);
  TPF_CUDA_TRY(cudaGetLastError());
  TPF_CUDA_TRY(cudaMemcpyAsync(zout, cur, bytes, cudaMemcpyDeviceToDevice, s));
  return TPF_OK;
}

int tpf_lppe_precondition(tpf_lppe* lp, const double* r, double* z, int smooth, double omega, void* stream) {
  TPF_CHECK_ARG(lp && r && z, "NULL argument");
  TPF_CHECK_ARG(lp->have_feat, "call tpf_lppe_prepare first");
  TPF_CHECK_ARG(smooth >= 0 && smooth <= 32, "smooth must be in [0, 32]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = tpf::unet_prepare_weights(lp->net, s);
  if (st) return st;
  TPF_CUDA_TRY(cudaMemcpyAsync(lp->r, r, sizeof(double) * lp->g.ndof, cudaMemcpyDeviceToDevice, s));
  rscale_partials_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(lp->g, lp->r, lp->part);
  rscale_finish_kernel<<<1, 256, 0, s>>>(lp->part, kRedBlocks, lp->g.ndof, lp->st);
  TPF_CUDA_TRY(cudaGetLastError());
  double* zr = nullptr;
  if ((st = enqueue_precond(lp, smooth, omega, s, &zr))) return st;
  TPF_CUDA_TRY(cudaMemcpyAsync(z, zr, sizeof(double) * lp->g.ndof, cudaMemcpyDeviceToDevice, s));
  return tpf::unet_check(lp->net, s);
}

int tpf_lppe_solve(tpf_lppe* lp, const double* rhs, const double* rho, double* p, const double* p_init,
                   const tpf_learned_options* opt, void* stream, tpf_lppe_result* result) {
  TPF_CHECK_ARG(lp && rhs && p, "NULL argument");
  tpf_learned_options o;
  if (opt) o = *opt; else tpf_lppe_default_options(&o);
  TPF_CHECK_ARG(o.tol > 0.0 && std::isfinite(o.tol), "tolerance must be > 0");
  TPF_CHECK_ARG(o.maxiter >= 0, "maxiter must be >= 0");
  TPF_CHECK_ARG(o.smooth >= 0 && o.smooth <= 32, "smooth must be in [0, 32]");
  TPF_CHECK_ARG(o.check_every >= 1 && o.check_every <= 1024, "check_every must be in [1, 1024]");
  TPF_CHECK_ARG(o.window >= 1 && o.window <= kMaxWin, "window must be in [1, %d]", kMaxWin);
  TPF_CHECK_ARG(o.outer == 0 || o.outer == 1, "outer must be 0 (flexible CG) or 1 (flexible GMRES)");
  TPF_CHECK_ARG(o.outer == 0 || (o.restart >= 1 && o.restart <= 128), "restart must be in [1, 128]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st;
  if (rho && (st = tpf_lppe_prepare(lp, rho, stream))) return st;
  if ((st = refresh_view(lp))) return st;
  TPF_CHECK_ARG(lp->v.prepared && lp->have_feat, "operator coefficients are not initialised (call prepare first)");
  tpf_lppe_result local{};
  tpf_lppe_result* res = result ? result : &local;
  *res = tpf_lppe_result{};
  if ((st = tpf::unet_prepare_weights(lp->net, s))) return st;
  lp->win = o.window;
  const LGrid& g = lp->g;
  fcg_init_kernel<<<ew_blocks(g.ndof), 256, 0, s>>>(g, rhs, p_init, lp->b, lp->x);

  if (o.outer == 1) {
    GmresOutcome out;
    if ((st = solve_fgmres(lp, o, s, p_init != nullptr, out))) return st;
    res->iterations = out.inner;
    res->restarts = out.inner > 0 ? (out.inner + o.restart - 1) / o.restart : 0;
    res->rel_residual = out.bnrm2 > 0.0 ? out.rnorm / out.bnrm2 : 0.0;
    copy_x_kernel<<<ew_blocks(g.ndof), 256, 0, s>>>(g.ndof, g.pin, lp->x, p);
    TPF_CUDA_TRY(cudaGetLastError());
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    if ((st = tpf::unet_check(lp->net, s))) return st;
    if (out.converged) {
      res->info = 0;
      return TPF_OK;
    }
    if (o.fallback) {
      tpf_ppe_options saved{}, po{};
      tpf::ppe_options(lp->ppe, &saved);
      po = saved;
      po.method = TPF_PPE_CG;
      po.precond = TPF_PRECOND_JACOBI;
      po.precision = TPF_PREC_F64;
      po.tol = o.tol;
      po.maxiter = std::max<int64_t>(o.maxiter, 20000);
      if ((st = tpf_ppe_set_options(lp->ppe, &po))) return st;
      tpf_ppe_result pr{};
      st = tpf_ppe_solve(lp->ppe, rhs, nullptr, p, p, stream, &pr);
      tpf_ppe_set_options(lp->ppe, &saved);
      res->fell_back = 1;
      res->fallback_iterations = pr.iterations;
      res->rel_residual = pr.rel_residual;
      res->info = pr.info;
      return st;
    }
    res->info = (int)std::min<long long>(o.maxiter, 0x7fffffff);
    tpf::set_error("learned flexible GMRES did not converge (info=%d)", res->info);
    return TPF_ENOCONV;
  }

  if ((st = true_residual(lp, s, o.tol, 1, o.window))) return st;
  if ((st = read_state(lp, s))) return st;
  bool converged = lp->st_host->done != 0;
  bool graph_ready = false;
  // stall: the best ||r|| has not fallen by stall_factor within stall_checks
  // checks (||r|| of CG-type methods is not monotone, so compare the best)
  double rr_ref = lp->st_host->rr;
  long long ref_iter = 0;
  bool stalled = false;
  while (!converged && lp->st_host->iters < o.maxiter) {
    const long long left = o.maxiter - lp->st_host->iters;
    const int chunk = (int)std::min<long long>(o.check_every, left);
    for (int k = 0; k < chunk; ++k) {
      if (o.use_graph && graph_ready) {
        TPF_CUDA_TRY(cudaGraphLaunch(lp->exec, s));
      } else {
        if ((st = enqueue_iteration(lp, o.smooth, o.omega, s))) return st;
      }
    }
    if ((st = read_state(lp, s))) return st;
    if (o.use_graph && !graph_ready) {
      // the eager chunk initialised every kernel attribute; capture from here on
      if ((st = build_graph(lp, o.smooth, o.omega))) return st;
      graph_ready = true;
    }
    if (lp->st_host->done) {
      // test convergence on the true residual; restart the recurrence from it otherwise
      if ((st = true_residual(lp, s, o.tol, 0, o.window))) return st;
      if ((st = read_state(lp, s))) return st;
      converged = lp->st_host->done != 0;
      rr_ref = lp->st_host->rr;
      ref_iter = lp->st_host->iters;
      continue;
    }
    const double rr = lp->st_host->rr;
    if (rr < o.stall_factor * o.stall_factor * rr_ref) {
      rr_ref = rr;
      ref_iter = lp->st_host->iters;
    }
    if (o.fallback && o.stall_checks > 0 &&
        lp->st_host->iters - ref_iter >= (long long)o.stall_checks * o.check_every) {
      stalled = true;
      break;
    }
  }
  res->iterations = lp->st_host->iters;
  res->restarts = lp->st_host->restarts;
  copy_x_kernel<<<ew_blocks(g.ndof), 256, 0, s>>>(g.ndof, g.pin, lp->x, p);
  TPF_CUDA_TRY(cudaGetLastError());
  if (converged) {
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    res->rel_residual = lp->st_host->bb > 0.0 ? std::sqrt(lp->st_host->rr / lp->st_host->bb) : 0.0;
    res->info = 0;
    return TPF_OK;
  }
  if (o.fallback && (stalled || lp->st_host->iters >= o.maxiter)) {
    // plain Jacobi PCG from the current iterate
    tpf_ppe_options saved{}, po{};
    tpf::ppe_options(lp->ppe, &saved);
    po = saved;
    po.method = TPF_PPE_CG;
    po.precond = TPF_PRECOND_JACOBI;
    po.precision = TPF_PREC_F64;
    po.tol = o.tol;
    po.maxiter = std::max<int64_t>(o.maxiter, 20000);
    if ((st = tpf_ppe_set_options(lp->ppe, &po))) return st;
    tpf_ppe_result pr{};
    st = tpf_ppe_solve(lp->ppe, rhs, nullptr, p, p, stream, &pr);
    tpf_ppe_set_options(lp->ppe, &saved);
    res->fell_back = 1;
    res->fallback_iterations = pr.iterations;
    res->rel_residual = pr.rel_residual;
    res->info = pr.info;
    return st;
  }
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  res->rel_residual = lp->st_host->bb > 0.0 ? std::sqrt(lp->st_host->rr / lp->st_host->bb) : 0.0;
  res->info = (int)std::min<long long>(o.maxiter, 0x7fffffff);
  tpf::set_error("learned flexible CG did not converge (info=%d)", res->info);
  return TPF_ENOCONV;
}

}  // extern "C"

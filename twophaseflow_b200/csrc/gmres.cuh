// Restarted GMRES on the device: SciPy 1.18.1's left-preconditioned gmres
// (scipy/sparse/linalg/_isolve/iterative.py) with its gh-8400 inner
// tolerance control, restated for CUDA.  The Hessenberg matrix, the Givens
// rotations and the residual vector live on the device; the host reads one
// small state block per restart cycle.  Classical Gram-Schmidt with a
// conditional re-orthogonalization pass stands in for SciPy's modified
// Gram-Schmidt (the same basis up to rounding).  An Arnoldi column is the
// caller's operator and preconditioner plus four kernels (gs1: first-pass
// inner products; gs2: the update and, without re-orthogonalization, the
// norm and the Givens step; gs3: the second pass when needed; the scaling of
// the new basis vector), each finishing its reductions in its last block.
// Every kernel of a column skips its work once the device-side state marks
// the cycle done, so a whole cycle (m columns) is captured once as a CUDA
// graph and replayed.
//
// The operator, the residual and the preconditioner are the caller's
// (functors enqueueing kernels on a stream): the FVM PPE (ppe.cu) and the
// FCCD PPE (fccd_ppe.cu) share this driver.
#pragma once

#include "tpf_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace {

// restart length limit of the fused kernels' shared staging (columns; the
// options accept restarts up to 1024)
constexpr int kGmMaxCols = 1024;

// ---- GMRES building blocks ---------------------------------------------------------

struct GmState {
  int done;          // inner loop finished (presid <= ptol or breakdown)
  int breakdown;
  int ncols;         // columns completed in this cycle
  int reorth;        // second Gram-Schmidt pass requested
  double presid;
  double ptol;
  double h0;         // ||w|| before orthogonalization
  double wn2;        // ||w||^2 scratch
  double rnorm;      // true residual norm (end of cycle)
  double scal;       // scale factor for the new basis vector
  unsigned int arrive;   // blocks finished in the current fused kernel (last-block reductions)
  int pad;
};

// partial dots: part[k*nb + block] = <V_k, w> for k < ncols, part[ncols*nb+block] = <w,w>
// Block partials of <V_k, w> for k < ncols and of <w, w> (k = ncols):
// part[k * nb + block].  The vectors are taken eight at a time in one sweep
// over w, with one block reduction per group (warp j reduces vector j of the
// group with the same shuffle tree a one-vector reduction uses).
__global__ void mdot_kernel(int ndof, const double* __restrict__ V, int ncols, const double* __restrict__ w,
                            double* part, const int* done) {
  if (done && *done) return;
  constexpr int KC = 8;   // vectors per sweep (<= warps per block)
  extern __shared__ double sh[];   // [KC][32]
  const int nb = gridDim.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k0 = 0; k0 <= ncols; k0 += KC) {
    double acc[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) acc[j] = 0.0;
    // two elements per trip: 18 independent loads in flight per thread
    const int stride = gridDim.x * blockDim.x;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    for (; idx + stride < ndof; idx += 2 * stride) {
      const double wa = w[idx], wb = w[idx + stride];
      double va[KC], vb[KC];
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        const int k = k0 + j;
        va[j] = (k < ncols) ? V[(size_t)k * ndof + idx] : wa;
        vb[j] = (k < ncols) ? V[(size_t)k * ndof + idx + stride] : wb;
      }
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        if (k0 + j <= ncols) {
          acc[j] += va[j] * wa;
          acc[j] += vb[j] * wb;
        }
      }
    }
    if (idx < ndof) {
      const double wi = w[idx];
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        const int k = k0 + j;
        if (k <= ncols) acc[j] += ((k < ncols) ? V[(size_t)k * ndof + idx] : wi) * wi;
      }
    }
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      const double v = tpf::warp_sum(acc[j]);
      if (lane == 0) sh[j * 32 + wid] = v;
    }
    __syncthreads();
    if (wid < KC && k0 + wid <= ncols) {
      double t = (lane < nw) ? sh[wid * 32 + lane] : 0.0;
      t = tpf::warp_sum(t);
      if (lane == 0) part[(size_t)(k0 + wid) * nb + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

// sum partials -> out[k] (k <= ncols); mode selects how the state uses them.
// mode 0: first GS pass (h column = dots, h0 = sqrt(<w,w>)), decide re-orth
// mode 1: second pass (h column += dots)
// mode 2: plain norm -> out[0] = sqrt(<w,w>)
// One block; warp j sums the partials of vectors j, j + nwarps, ... (lane l:
// blocks l, l + 32, ..., then a shuffle tree), so all vectors are summed at
// once; thread 0 then applies the mode's scalar logic in vector order.
__global__ void mdot_finalize_kernel(const double* part, int nb, int ncols, double* hcol, GmState* st,
                                     int mode, double* out_norm) {
  if (mode != 2 && st->done) return;
  if (mode == 1 && !st->reorth) return;
  extern __shared__ double sums[];   // [ncols + 1]
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = wid; k <= ncols; k += nw) {
    double acc = 0.0;
    for (int b = lane; b < nb; b += 32) acc += part[(size_t)k * nb + b];
    acc = tpf::warp_sum(acc);
    if (lane == 0) sums[k] = acc;
  }
  __syncthreads();
  if (mode == 2) {
    if (threadIdx.x == 0) *out_norm = sqrt(sums[0]);
    return;
  }
  if (mode == 1) {
    for (int k = threadIdx.x; k < ncols; k += blockDim.x) hcol[k] += sums[k];
    if (threadIdx.x == 0) st->wn2 = 0.0;
    return;
  }
  for (int k = threadIdx.x; k < ncols; k += blockDim.x) hcol[k] = sums[k];
  if (threadIdx.x == 0) {
    const double sw = sums[ncols];
    st->h0 = sqrt(sw);
    double proj = 0.0;
    for (int q = 0; q < ncols; ++q) proj += sums[q] * sums[q];
    st->reorth = (sw - proj < 0.5 * sw) ? 1 : 0;
  }
}

// Givens rotation generator for real (f, g): c f + s g = r, -s f + c g = 0,
// r carries the sign of f (the convention of LAPACK's lartg).
__device__ void givens_rot(double f, double g, double& c, double& s, double& r) {
  if (g == 0.0) { c = 1.0; s = 0.0; r = f; return; }
  if (f == 0.0) { c = 0.0; s = (g > 0.0) ? 1.0 : -1.0; r = fabs(g); return; }
  double d = hypot(f, g);
  c = fabs(f) / d;
  r = copysign(d, f);
  s = g / r;
}

__global__ void gm_scale_kernel(int ndof, const double* w, double* vout, const GmState* st) {
  tpf::chain_begin();
  if (st->done && st->scal == 0.0) return;
  // executed even when this column set done (the vector is then unused)
  const double sc = st->scal;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x)
    vout[idx] = w[idx] * sc;
  tpf::chain_end();
}

// y = H(:ncols,:ncols)^-1 S (SciPy's trsv loop), then coef = y
// Column-oriented back substitution R y = S (SciPy's order): y lives in
// shared memory and the updates y[q] -= y[k] R[k][q] of one column k run on
// the block's threads, one q each; every y[q] receives the same updates in
// the same order as a single thread would apply them (same bits).
__global__ void gm_backsolve_kernel(const double* H, int ldh, double* S, double* y, const GmState* st) {
  __shared__ double ys[kGmMaxCols + 1];
  const int col = st->ncols - 1;
  if (col < 0) return;
  for (int k = threadIdx.x; k <= col; k += blockDim.x) ys[k] = S[k];
  __syncthreads();
  if (threadIdx.x == 0 && H[(size_t)col * ldh + col] == 0.0) {
    S[col] = 0.0;
    ys[col] = 0.0;
  }
  __syncthreads();
  for (int k = col; k > 0; --k) {
    if (ys[k] != 0.0) {   // the same value in every thread: a uniform branch
      __syncthreads();
      if (threadIdx.x == 0) ys[k] /= H[(size_t)k * ldh + k];
      __syncthreads();
      const double t = ys[k];
      for (int q = threadIdx.x; q < k; q += blockDim.x) ys[q] -= t * H[(size_t)k * ldh + q];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && ys[0] != 0.0) ys[0] /= H[0];
  __syncthreads();
  for (int k = threadIdx.x; k <= col; k += blockDim.x) y[k] = ys[k];
}

__global__ void gm_update_x_kernel(int ndof, const double* __restrict__ V, const double* y, double* x,
                                   const GmState* st) {
  int ncols = st->ncols;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int k = 0; k < ncols; ++k) acc += y[k] * V[(size_t)k * ndof + idx];
    x[idx] += acc;
  }
}

__global__ void gm_start_kernel(int ndof, const double* w, double* v0, double* S, int m1, GmState* st,
                                double vnorm, double ptol) {
  const double inv = 1.0 / vnorm;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x)
    v0[idx] = w[idx] * inv;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int k = 0; k < m1; ++k) S[k] = 0.0;
    S[0] = vnorm;
    st->done = 0;
    st->breakdown = 0;
    st->ncols = 0;
    st->reorth = 0;
    st->ptol = ptol;
    st->presid = 0.0;
  }
}


// ---- fused Gram-Schmidt kernels (one column = operator, preconditioner, gs1,
// gs2, gs3, scale) ------------------------------------------------------------------
//
// Block partials of <V_k, w> (k < nv, slot nv - 1 may be <w, w>) accumulated
// eight vectors per sweep as in mdot_kernel; the last block to finish sums
// the partials in block order (fixed tree) and applies the column's scalar
// logic, so no separate finalize launch is needed.

__device__ __forceinline__ bool gm_last_block(GmState* st) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&st->arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (s_last) __threadfence();
  return s_last != 0;
}

// partials of <V_k, w> for k < nv; with_ww: slot nv is <w, w>
__device__ __forceinline__ void gm_partials(int ndof, const double* __restrict__ V, int nv, bool with_ww,
                                            const double* w, double* part, double* sh) {
  constexpr int KC = 8;
  const int nb = gridDim.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int ntot = nv + (with_ww ? 1 : 0);
  for (int k0 = 0; k0 < ntot; k0 += KC) {
    double acc[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) acc[j] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += stride) {
      const double wi = w[idx];
#pragma unroll
      for (int j = 0; j < KC; ++j) {
        const int k = k0 + j;
        if (k < ntot) acc[j] += ((k < nv) ? V[(size_t)k * ndof + idx] : wi) * wi;
      }
    }
#pragma unroll
    for (int j = 0; j < KC; ++j) {
      const double v = tpf::warp_sum(acc[j]);
      if (lane == 0) sh[j * 32 + wid] = v;
    }
    __syncthreads();
    if (wid < KC && k0 + wid < ntot) {
      double t = (lane < nw) ? sh[wid * 32 + lane] : 0.0;
      t = tpf::warp_sum(t);
      if (lane == 0) part[(size_t)(k0 + wid) * nb + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

// sums of partial slots [0, ntot) in block order into out[] (last block only)
__device__ __forceinline__ void gm_sum_partials(const double* part, int nb, int ntot, double* out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = wid; k < ntot; k += nw) {
    double acc = 0.0;
    for (int b = lane; b < nb; b += 32) acc += __ldcg(part + (size_t)k * nb + b);
    acc = tpf::warp_sum(acc);
    if (lane == 0) out[k] = acc;
  }
  __syncthreads();
}

// The column's scalar step (gm_column_kernel's arithmetic), run by the last
// block of gs2 / gs3 with the column staged in shared memory.
__device__ void gm_column_step(double* H, int ldh, double* givens, double* S, GmState* st, int col, double h1,
                               const double* hcol2, double* shc) {
  double* hc = H + (size_t)col * ldh;
  double* sg = shc + col + 2;
  const bool reorth = st->reorth != 0;
  for (int k = threadIdx.x; k <= col; k += blockDim.x) {
    double v = __ldcg(hc + k);
    if (reorth) v += __ldcg(hcol2 + k);
    shc[k] = v;
  }
  for (int k = threadIdx.x; k < 2 * col; k += blockDim.x) sg[k] = __ldcg(givens + k);
  __syncthreads();
  if (threadIdx.x == 0) {
    const double eps = 2.220446049250313e-16;
    shc[col + 1] = h1;
    int breakdown = 0;
    if (h1 <= eps * st->h0) {
      shc[col + 1] = 0.0;
      breakdown = 1;
      st->scal = 1.0;
    } else {
      st->scal = 1.0 / h1;
    }
    for (int k = 0; k < col; ++k) {
      const double c = sg[2 * k], sn = sg[2 * k + 1];
      const double n0 = shc[k], n1 = shc[k + 1];
      shc[k] = c * n0 + sn * n1;
      shc[k + 1] = -sn * n0 + c * n1;
    }
    double c, sn, mag;
    givens_rot(shc[col], shc[col + 1], c, sn, mag);
    givens[2 * col] = c;
    givens[2 * col + 1] = sn;
    shc[col] = mag;
    shc[col + 1] = 0.0;
    const double t = -sn * S[col];
    S[col] = c * S[col];
    S[col + 1] = t;
    st->presid = fabs(t);
    st->ncols = col + 1;
    st->breakdown = breakdown;
    if (st->presid <= st->ptol || breakdown) st->done = 1;
  }
  __syncthreads();
  for (int k = threadIdx.x; k <= col + 1; k += blockDim.x) hc[k] = shc[k];
}

// gs1: <V_k, w> (k <= col) and <w, w>; last block: H column = the dots,
// h0 = ||w||, the re-orthogonalization decision, hcol2 = 0
__global__ void gs1_kernel(int ndof, const double* __restrict__ V, int col, const double* __restrict__ w,
                           double* part, double* hcol, double* hcol2, GmState* st) {
  tpf::chain_begin();
  if (st->done) return;
  __shared__ double sh[8 * 32];
  __shared__ double sums[kGmMaxCols + 2];
  gm_partials(ndof, V, col + 1, true, w, part, sh);
  if (!gm_last_block(st)) return;
  gm_sum_partials(part, gridDim.x, col + 2, sums);
  for (int k = threadIdx.x; k <= col; k += blockDim.x) {
    hcol[k] = sums[k];
    hcol2[k] = 0.0;
  }
  if (threadIdx.x == 0) {
    const double sw = sums[col + 1];
    st->h0 = sqrt(sw);
    double proj = 0.0;
    for (int q = 0; q <= col; ++q) proj += sums[q] * sums[q];
    st->reorth = (sw - proj < 0.5 * sw) ? 1 : 0;
    st->arrive = 0u;
  }
  tpf::chain_end();
}

// gs2: w -= sum_k hcol_k V_k; then either the second pass's dots
// (re-orthogonalization: last block -> hcol2) or ||w|| and the column step
__global__ void gs2_kernel(int ndof, const double* __restrict__ V, int col, double* w, const double* hcol,
                           double* part, double* H, int ldh, double* givens, double* S, double* hcol2, GmState* st) {
  tpf::chain_begin();
  if (st->done) return;
  __shared__ double sh[8 * 32];
  __shared__ double sums[3 * kGmMaxCols + 4];
  const bool reorth = st->reorth != 0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x) {
    double acc = w[idx];
#pragma unroll 8
    for (int k = 0; k <= col; ++k) acc -= hcol[k] * V[(size_t)k * ndof + idx];
    w[idx] = acc;
  }
  if (reorth) gm_partials(ndof, V, col + 1, false, w, part, sh);
  else gm_partials(ndof, V, 0, true, w, part, sh);
  if (!gm_last_block(st)) return;
  if (reorth) {
    gm_sum_partials(part, gridDim.x, col + 1, sums);
    for (int k = threadIdx.x; k <= col; k += blockDim.x) hcol2[k] = sums[k];
    if (threadIdx.x == 0) st->arrive = 0u;
    return;
  }
  gm_sum_partials(part, gridDim.x, 1, sums);
  const double h1 = sqrt(sums[0]);
  __syncthreads();
  gm_column_step(H, ldh, givens, S, st, col, h1, hcol2, sums);
  if (threadIdx.x == 0) st->arrive = 0u;
  tpf::chain_end();
}

// gs3 (re-orthogonalization only): w -= sum_k hcol2_k V_k; ||w||; column step
__global__ void gs3_kernel(int ndof, const double* __restrict__ V, int col, double* w, double* part, double* H,
                           int ldh, double* givens, double* S, const double* hcol2, GmState* st) {
  tpf::chain_begin();
  if (st->done || !st->reorth) return;
  __shared__ double sh[8 * 32];
  __shared__ double sums[3 * kGmMaxCols + 4];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ndof; idx += gridDim.x * blockDim.x) {
    double acc = w[idx];
#pragma unroll 8
    for (int k = 0; k <= col; ++k) acc -= hcol2[k] * V[(size_t)k * ndof + idx];
    w[idx] = acc;
  }
  gm_partials(ndof, V, 0, true, w, part, sh);
  if (!gm_last_block(st)) return;
  gm_sum_partials(part, gridDim.x, 1, sums);
  const double h1 = sqrt(sums[0]);
  __syncthreads();
  gm_column_step(H, ldh, givens, S, st, col, h1, hcol2, sums);
  if (threadIdx.x == 0) st->arrive = 0u;
  tpf::chain_end();
}

// Device GMRES workspace of one solver handle.  V holds restart_cap + 1
// basis vectors; gm holds H (restart_cap x (restart_cap + 2)), the Givens
// pairs, S, y, two Hessenberg columns and two norms; part holds the block
// partial sums (at least 2 x blocks doubles).  exec / cap / key persist per
// handle: the captured cycle graph, the private capture stream and the key
// of what the graph's launches depend on.
struct GmresWork {
  int n = 0;
  int ew_blocks = 0;
  int part_len = 0;
  int restart_cap = 0;
  double* V = nullptr;
  double* gm = nullptr;
  double* part = nullptr;
  GmState* gst = nullptr;
  double* b = nullptr;     // right-hand side (prepared by the caller)
  double* x = nullptr;     // iterate (x0 set by the caller)
  double* r = nullptr;     // residual scratch
  double* w = nullptr;     // preconditioned-vector scratch
  double* t = nullptr;     // operator-output scratch
  cudaGraphExec_t* exec = nullptr;
  cudaStream_t* cap = nullptr;
  long long* key = nullptr;   // 6 entries
};

inline int gm_norm2(const GmresWork& W, const double* v, double* out, cudaStream_t s) {
  const int nb = std::min(W.ew_blocks, W.part_len / 2);
  mdot_kernel<<<nb, 256, 8 * 32 * sizeof(double), s>>>(W.n, nullptr, 0, v, W.part, nullptr);
  mdot_finalize_kernel<<<1, 1024, sizeof(double), s>>>(W.part, nb, 0, nullptr, W.gst, 2, out);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

inline int gm_read_scalar(const double* dev, double* host, cudaStream_t s) {
  TPF_CUDA_TRY(cudaMemcpyAsync(host, dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  return TPF_OK;
}

struct GmresOutcome {
  long long inner = 0;     // Arnoldi columns (SciPy's inner iterations)
  long long applies = 0;   // operator applications
  double bnrm2 = 0.0;
  double rnorm = 0.0;      // true residual norm at exit
  bool converged = false;
  bool stalled = false;    // flexible GMRES: stopped by its stall rule
};

// SciPy gmres(A, b, x0, rtol=tol, atol=0, restart, maxiter, M) on the
// device.  apply(in, out, stream, done): out = A in; resid(x, r, stream):
// r = b - A x; precond(in, out, stream, done): out = M in.  Kernels given a
// non-null `done` may skip their work once *done is set.  W.b and W.x
// (x0; x_nonzero says whether it is nonzero) are set by the caller; on
// return W.x holds the iterate.  key_a / key_b: the caller's part of the
// cycle graph's key (what its operator launches depend on besides the
// buffers).
template <class Apply, class Resid, class Precond>
int gmres_solve(GmresWork& W, int restart, double tol, long long maxiter, bool x_nonzero, long long key_a,
                long long key_b, Apply apply, Resid resid, Precond precond, cudaStream_t s, GmresOutcome& out) {
  const int n = W.n;
  int st;
  const int m = std::min(restart, n);
  const int ldh = W.restart_cap + 2;
  double* H = W.gm;
  double* givens = H + (size_t)W.restart_cap * ldh;
  double* S = givens + 2 * W.restart_cap;
  double* y = S + (W.restart_cap + 1);
  double* hcol = y + (W.restart_cap + 1);
  double* hcol2 = hcol + (W.restart_cap + 1);
  double* wnorm = hcol2 + (W.restart_cap + 1);
  double* bnorm_d = wnorm + 1;
  (void)hcol;
  TPF_CUDA_TRY(cudaMemsetAsync(H, 0, sizeof(double) * (size_t)W.restart_cap * ldh, s));
  TPF_CUDA_TRY(cudaMemsetAsync(W.gst, 0, sizeof(GmState), s));
  if ((st = gm_norm2(W, W.b, bnorm_d, s))) return st;
  double bnrm2 = 0.0;
  if ((st = gm_read_scalar(bnorm_d, &bnrm2, s))) return st;
  out = GmresOutcome{};
  out.bnrm2 = bnrm2;
  if (bnrm2 == 0.0) {
    TPF_CUDA_TRY(cudaMemsetAsync(W.x, 0, sizeof(double) * n, s));
    out.converged = true;
    return TPF_OK;
  }
  const double atol = tol * bnrm2;
  const double eps = 2.220446049250313e-16;
  // Mb_nrm2 = ||M b||
  if ((st = precond(W.b, W.w, s, nullptr))) return st;
  if ((st = gm_norm2(W, W.w, wnorm, s))) return st;
  double Mb_nrm2 = 0.0;
  if ((st = gm_read_scalar(wnorm, &Mb_nrm2, s))) return st;
  double ptol_max_factor = 1.0;
  double ptol = Mb_nrm2 * std::min(ptol_max_factor, atol / bnrm2);
  double presid = 0.0, rnorm = INFINITY;
  // four blocks per SM for the basis dot products: enough loads in flight,
  // few partials to sum per vector
  const int nb_dot = std::min(std::min(W.ew_blocks, W.part_len / (m + 2)), std::max(1, 4 * tpf::sm_count()));
  const int* done = &W.gst->done;
  bool converged = false;
  long long applies = 0, inner = 0;
  auto enqueue_cycle = [&](cudaStream_t cs) -> int {
    int est;
    for (int col = 0; col < m; ++col) {
      const double* vc = W.V + (size_t)col * n;
      if ((est = apply(vc, W.t, cs, done))) return est;
      if ((est = precond(W.t, W.w, cs, done))) return est;
      double* hc = H + (size_t)col * ldh;
      tpf::launch_chained(gs1_kernel, nb_dot, 256, 0, cs, n, W.V, col, W.w, W.part, hc, hcol2, W.gst);
      tpf::launch_chained(gs2_kernel, nb_dot, 256, 0, cs, n, W.V, col, W.w, hc, W.part, H, ldh, givens, S, hcol2,
                          W.gst);
      tpf::launch_chained(gs3_kernel, nb_dot, 256, 0, cs, n, W.V, col, W.w, W.part, H, ldh, givens, S, hcol2, W.gst);
      tpf::launch_chained(gm_scale_kernel, W.ew_blocks, 256, 0, cs, n, W.w, W.V + (size_t)(col + 1) * n, W.gst);
      TPF_CUDA_TRY(cudaGetLastError());
    }
    return TPF_OK;
  };
  const long long key[6] = {(long long)m, (long long)nb_dot, key_a, key_b, (long long)(intptr_t)W.V, (long long)n};
  for (long long iteration = 0; iteration < maxiter; ++iteration) {
    if (iteration == 0) {
      if (x_nonzero) {
        if ((st = resid(W.x, W.r, s))) return st;
        ++applies;
      } else {
        TPF_CUDA_TRY(cudaMemcpyAsync(W.r, W.b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      }
      if ((st = gm_norm2(W, W.r, wnorm, s))) return st;
      double r0 = 0.0;
      if ((st = gm_read_scalar(wnorm, &r0, s))) return st;
      if (r0 < atol) { rnorm = r0; converged = true; break; }
    }
    // v0 = M r / ||M r||
    TPF_CUDA_TRY(cudaMemsetAsync(W.gst, 0, sizeof(int), s));  // done = 0 for the precond call
    if ((st = precond(W.r, W.w, s, nullptr))) return st;
    if ((st = gm_norm2(W, W.w, wnorm, s))) return st;
    double v0n = 0.0;
    if ((st = gm_read_scalar(wnorm, &v0n, s))) return st;
    gm_start_kernel<<<W.ew_blocks, 256, 0, s>>>(n, W.w, W.V, S, m + 1, W.gst, v0n, ptol);
    if (!*W.exec || std::memcmp(W.key, key, sizeof(key)) != 0) {
      if (*W.exec) { cudaGraphExecDestroy(*W.exec); *W.exec = nullptr; }
      // captured on a private stream (the caller's may be the legacy default
      // stream, which cannot be captured); replayed on the caller's
      if (!*W.cap && cudaStreamCreateWithFlags(W.cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        *W.cap = nullptr;
        tpf::set_error("cudaStreamCreate failed");
        return TPF_ECUDA;
      }
      TPF_CUDA_TRY(cudaStreamBeginCapture(*W.cap, cudaStreamCaptureModeThreadLocal));
      const int cst = enqueue_cycle(*W.cap);
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(*W.cap, &graph);
      if (cst || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (cst) return cst;
        tpf::set_error("capturing the GMRES cycle failed: %s", cudaGetErrorString(ce));
        return TPF_ECUDA;
      }
      const cudaError_t ie = cudaGraphInstantiate(W.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        *W.exec = nullptr;
        cudaGetLastError();
        tpf::set_error("instantiating the GMRES cycle graph failed: %s", cudaGetErrorString(ie));
        return TPF_ECUDA;
      }
      std::memcpy(W.key, key, sizeof(key));
    }
    TPF_CUDA_TRY(cudaGraphLaunch(*W.exec, s));
    GmState hs{};
    TPF_CUDA_TRY(cudaMemcpyAsync(&hs, W.gst, sizeof(GmState), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    inner += hs.ncols;
    applies += hs.ncols;
    presid = hs.presid;
    gm_backsolve_kernel<<<1, 128, 0, s>>>(H, ldh, S, y, W.gst);
    gm_update_x_kernel<<<W.ew_blocks, 256, 0, s>>>(n, W.V, y, W.x, W.gst);
    if ((st = resid(W.x, W.r, s))) return st;
    ++applies;
    if ((st = gm_norm2(W, W.r, wnorm, s))) return st;
    if ((st = gm_read_scalar(wnorm, &rnorm, s))) return st;
    if (rnorm <= atol) { converged = true; break; }
    if (hs.breakdown) break;
    if (presid <= ptol) ptol_max_factor = std::max(eps, 0.25 * ptol_max_factor);
    else ptol_max_factor = std::min(1.0, 1.5 * ptol_max_factor);
    ptol = presid * std::min(ptol_max_factor, atol / rnorm);
  }
  out.inner = inner;
  out.applies = applies;
  out.rnorm = rnorm;
  out.converged = converged;
  return TPF_OK;
}

}  // namespace

namespace {

// Flexible restarted GMRES (Saad, "A flexible inner-outer preconditioned
// GMRES algorithm", SIAM J. Sci. Comput. 14, 1993): right preconditioning by
// a preconditioner that may change from column to column (a network), so
// z_j = M_j(v_j) is kept in Z (restart columns of n), w = A z_j is
// orthogonalized against V with the same column kernels as gmres_solve, and
// a cycle ends with x += Z y.  The Givens estimate is then the
// unpreconditioned residual norm, so a cycle stops once it meets tol ||b||;
// each restart starts from the true residual r = b - A x.
// apply / resid / precond as for gmres_solve; Z: restart * n doubles.
// Stall rule (stall_iters > 0): after a cycle, the best true ||r|| so far has
// not fallen below stall_factor times the reference value within stall_iters
// Arnoldi columns -> stop with out.stalled (the reference value is reset
// whenever it does fall that far).
template <class Apply, class Resid, class Precond>
int fgmres_solve(GmresWork& W, double* Z, int restart, double tol, long long maxiter, bool x_nonzero,
                 long long key_a, long long key_b, Apply apply, Resid resid, Precond precond, cudaStream_t s,
                 GmresOutcome& out, double stall_factor = 0.5, long long stall_iters = 0) {
  const int n = W.n;
  int st;
  const int m = std::min(restart, n);
  const int ldh = W.restart_cap + 2;
  double* H = W.gm;
  double* givens = H + (size_t)W.restart_cap * ldh;
  double* S = givens + 2 * W.restart_cap;
  double* y = S + (W.restart_cap + 1);
  double* hcol = y + (W.restart_cap + 1);
  double* hcol2 = hcol + (W.restart_cap + 1);
  double* wnorm = hcol2 + (W.restart_cap + 1);
  double* bnorm_d = wnorm + 1;
  TPF_CUDA_TRY(cudaMemsetAsync(H, 0, sizeof(double) * (size_t)W.restart_cap * ldh, s));
  TPF_CUDA_TRY(cudaMemsetAsync(W.gst, 0, sizeof(GmState), s));
  if ((st = gm_norm2(W, W.b, bnorm_d, s))) return st;
  double bnrm2 = 0.0;
  if ((st = gm_read_scalar(bnorm_d, &bnrm2, s))) return st;
  out = GmresOutcome{};
  out.bnrm2 = bnrm2;
  if (bnrm2 == 0.0) {
    TPF_CUDA_TRY(cudaMemsetAsync(W.x, 0, sizeof(double) * n, s));
    out.converged = true;
    return TPF_OK;
  }
  const double atol = tol * bnrm2;
  const int nb_dot = std::min(std::min(W.ew_blocks, W.part_len / (m + 2)), std::max(1, 4 * tpf::sm_count()));
  const int* done = &W.gst->done;
  auto enqueue_cycle = [&](cudaStream_t cs) -> int {
    int est;
    for (int col = 0; col < m; ++col) {
      const double* vc = W.V + (size_t)col * n;
      double* zc = Z + (size_t)col * n;
      if ((est = precond(vc, zc, cs, done))) return est;
      if ((est = apply(zc, W.w, cs, done))) return est;
      double* hc = H + (size_t)col * ldh;
      tpf::launch_chained(gs1_kernel, nb_dot, 256, 0, cs, n, W.V, col, W.w, W.part, hc, hcol2, W.gst);
      tpf::launch_chained(gs2_kernel, nb_dot, 256, 0, cs, n, W.V, col, W.w, hc, W.part, H, ldh, givens, S, hcol2,
                          W.gst);
      tpf::launch_chained(gs3_kernel, nb_dot, 256, 0, cs, n, W.V, col, W.w, W.part, H, ldh, givens, S, hcol2, W.gst);
      tpf::launch_chained(gm_scale_kernel, W.ew_blocks, 256, 0, cs, n, W.w, W.V + (size_t)(col + 1) * n, W.gst);
      TPF_CUDA_TRY(cudaGetLastError());
    }
    return TPF_OK;
  };
  // -m marks the flexible cycle (a different graph from gmres_solve's)
  const long long key[6] = {-(long long)m, (long long)nb_dot, key_a, key_b, (long long)(intptr_t)Z, (long long)n};
  long long applies = 0, inner = 0;
  double rnorm = INFINITY;
  bool converged = false;
  if (x_nonzero) {
    if ((st = resid(W.x, W.r, s))) return st;
    ++applies;
  } else {
    TPF_CUDA_TRY(cudaMemcpyAsync(W.r, W.b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  }
  if ((st = gm_norm2(W, W.r, wnorm, s))) return st;
  if ((st = gm_read_scalar(wnorm, &rnorm, s))) return st;
  double ref_rnorm = rnorm;
  long long ref_inner = 0;
  for (long long iteration = 0; iteration < maxiter && !converged; ++iteration) {
    if (rnorm <= atol) { converged = true; break; }
    gm_start_kernel<<<W.ew_blocks, 256, 0, s>>>(n, W.r, W.V, S, m + 1, W.gst, rnorm, atol);
    if (!*W.exec || std::memcmp(W.key, key, sizeof(key)) != 0) {
      if (*W.exec) { cudaGraphExecDestroy(*W.exec); *W.exec = nullptr; }
      if (!*W.cap && cudaStreamCreateWithFlags(W.cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        *W.cap = nullptr;
        tpf::set_error("cudaStreamCreate failed");
        return TPF_ECUDA;
      }
      TPF_CUDA_TRY(cudaStreamBeginCapture(*W.cap, cudaStreamCaptureModeThreadLocal));
      const int cst = enqueue_cycle(*W.cap);
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(*W.cap, &graph);
      if (cst || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (cst) return cst;
        tpf::set_error("capturing the flexible GMRES cycle failed: %s", cudaGetErrorString(ce));
        return TPF_ECUDA;
      }
      const cudaError_t ie = cudaGraphInstantiate(W.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        *W.exec = nullptr;
        cudaGetLastError();
        tpf::set_error("instantiating the flexible GMRES cycle graph failed: %s", cudaGetErrorString(ie));
        return TPF_ECUDA;
      }
      std::memcpy(W.key, key, sizeof(key));
    }
    TPF_CUDA_TRY(cudaGraphLaunch(*W.exec, s));
    GmState hs{};
    TPF_CUDA_TRY(cudaMemcpyAsync(&hs, W.gst, sizeof(GmState), cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaStreamSynchronize(s));
    inner += hs.ncols;
    applies += hs.ncols;
    gm_backsolve_kernel<<<1, 128, 0, s>>>(H, ldh, S, y, W.gst);
    gm_update_x_kernel<<<W.ew_blocks, 256, 0, s>>>(n, Z, y, W.x, W.gst);
    if ((st = resid(W.x, W.r, s))) return st;
    ++applies;
    if ((st = gm_norm2(W, W.r, wnorm, s))) return st;
    if ((st = gm_read_scalar(wnorm, &rnorm, s))) return st;
    if (rnorm <= atol) converged = true;
    if (hs.breakdown) break;
    if (!converged && stall_iters > 0) {
      if (rnorm < stall_factor * ref_rnorm) {
        ref_rnorm = rnorm;
        ref_inner = inner;
      } else if (inner - ref_inner >= stall_iters) {
        out.stalled = true;
        break;
      }
    }
  }
  out.inner = inner;
  out.applies = applies;
  out.rnorm = rnorm;
  out.converged = converged;
  return TPF_OK;
}

}  // namespace

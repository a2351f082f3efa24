// CLS transport: the FCCD flux-form advection right-hand side and the TVD-RK3
// stages around it.
// Reference: src/twophase/ccd/fccd.py:213-233 (face slices), :279-299 (face
// value), :464-520 (face divergence), ccd/fccd_advection_helpers.py:8-72
// (flux contribution and the composed right-hand side),
// time_integration/tvd_rk3.py:26-48 (stages), levelset/fccd_advection.py:86-129
// (clip + periodic image after every stage), core/boundary.py:116-133 (image
// nodes).  Arithmetic uses explicit round-to-nearest operations in the order
// NumPy evaluates the reference's expressions (no fused multiply-add), so the
// results equal the reference's for the same CCD second derivatives.
#include "tpf_common.cuh"

#include <algorithm>

namespace {

__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }

inline int blocks_for(int64_t n, int per_sm) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)tpf::sm_count() * per_sm));
}

template <typename T>
__global__ void product_kernel(int64_t n, const T* a, const T* b, T* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (T)rn_mul((double)a[i], (double)b[i]);
}

struct FluxArgs {
  const void* prod;   // u_k * phi at the nodes
  const void* q;      // its CCD second derivative along the axis
  void* acc;
  int64_t outer, n, inner;
  double inv_h, h2_16;
  int periodic, accumulate;
  const double* wf;   // non-uniform: H_f^2 / 16 per face f (else h2_16)
  const double* wn;   // non-uniform: 1 / node width per node (wall: nodes 1..N-1 at k-1; periodic: N) (else inv_h)
};

template <typename T>
__device__ __forceinline__ double ldv(const void* p, int64_t i) { return (double)static_cast<const T*>(p)[i]; }

// face value between nodes j and j+1 (fccd.py:279-299):
// 0.5 (u_j + u_{j+1}) - (H^2/16) (q_j + q_{j+1})
template <typename T>
__device__ __forceinline__ double face_val(const FluxArgs& a, int64_t il, int64_t ir, int64_t f) {
  const double c = a.wf ? a.wf[f] : a.h2_16;
  return rn_sub(rn_mul(0.5, rn_add(ldv<T>(a.prod, il), ldv<T>(a.prod, ir))),
                rn_mul(c, rn_add(ldv<T>(a.q, il), ldv<T>(a.q, ir))));
}

// 1 / width of node k (periodic: the unique node k; wall: interior node k)
__device__ __forceinline__ double node_inv_w(const FluxArgs& a, int64_t k) {
  if (!a.wn) return a.inv_h;
  return a.periodic ? a.wn[k] : a.wn[k - 1];
}

template <typename T>
__device__ __forceinline__ void flux_store(const FluxArgs& a, int64_t idx, double div) {
  T* acc = static_cast<T*>(a.acc);
  const double c = -div;   // the contribution is minus the face divergence
  acc[idx] = (T)(a.accumulate ? rn_add((double)acc[idx], c) : rn_add(0.0, c));
}

// divergence at node k of the line starting at base (fccd.py:464-520):
// periodic: (F[k] - F[k-1]) / H over the N unique nodes (F[-1] = F[N-1], the
// face after node N-1 wraps to node 0), node N repeats node 0; wall: nodes
// 1..N-1, 0 on the wall nodes.
template <typename T>
__device__ __forceinline__ double flux_div_node(const FluxArgs& a, int64_t base, int64_t k) {
  const int64_t N = a.n - 1, s = a.inner;
  if (a.periodic) {
    const int64_t kk = (k == N) ? 0 : k;
    const int64_t kp = (kk == N - 1) ? 0 : kk + 1, km = (kk == 0) ? N - 1 : kk - 1;
    const double fr = face_val<T>(a, base + kk * s, base + kp * s, kk);
    const double fl = face_val<T>(a, base + km * s, base + kk * s, km);
    return rn_mul(rn_sub(fr, fl), node_inv_w(a, kk));
  }
  if (k == 0 || k == N) return 0.0;
  const double fr = face_val<T>(a, base + k * s, base + (k + 1) * s, k);
  const double fl = face_val<T>(a, base + (k - 1) * s, base + k * s, k - 1);
  return rn_mul(rn_sub(fr, fl), node_inv_w(a, k));
}

// one thread per node (contiguous or short-stride axes: the neighbours are in
// the same cache lines)
template <typename T>
__global__ void flux_div_kernel(FluxArgs a) {
  const int64_t tot = a.outer * a.n * a.inner;
  const bool small = tot < (int64_t(1) << 31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t k, in;
    if (small) {
      const uint32_t ii = (uint32_t)i, inn = (uint32_t)a.inner;
      in = ii % inn;
      k = (ii / inn) % (uint32_t)a.n;
    } else {
      in = i % a.inner;
      k = (i / a.inner) % a.n;
    }
    const int64_t base = i - k * a.inner;
    (void)in;
    flux_store<T>(a, i, flux_div_node<T>(a, base, k));
  }
}

// strided axes: thread (chunk, line) marches over a chunk of one line,
// consecutive threads on consecutive lines (coalesced), one face formed per
// node, the next node's operands loaded before the store
template <typename T>
__global__ void __launch_bounds__(256) flux_march_kernel(FluxArgs a, int64_t chunk, int64_t nchunks) {
  const int64_t lines = a.outer * a.inner, N = a.n - 1, s = a.inner;
  const int64_t work = lines * nchunks;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < work; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t qi = t / lines, c = t - qi * lines;
    const int64_t o = c / s, in = c - o * s;
    const int64_t base = o * a.n * s + in;
    const int64_t k0 = qi * chunk, k1 = min(k0 + chunk, a.n);
    if (a.periodic) {
      // face to the left of node k (k = N reads node 0's faces)
      auto fleft = [&](int64_t k) {
        const int64_t kk = (k == N) ? 0 : k;
        const int64_t km = (kk == 0) ? N - 1 : kk - 1;
        return face_val<T>(a, base + km * s, base + kk * s, km);
      };
      double fl = fleft(k0);
      for (int64_t k = k0; k < k1; ++k) {
        const int64_t kk = (k == N) ? 0 : k;
        const int64_t kp = (kk == N - 1) ? 0 : kk + 1;
        const double fr = (k == N) ? face_val<T>(a, base, base + kp * s, 0) : face_val<T>(a, base + kk * s, base + kp * s, kk);
        const double old = a.accumulate ? (double)static_cast<const T*>(a.acc)[base + k * s] : 0.0;
        const double flk = (k == N) ? fleft(N) : fl;
        const double c2 = -rn_mul(rn_sub(fr, flk), node_inv_w(a, kk));
        static_cast<T*>(a.acc)[base + k * s] = (T)rn_add(old, c2);
        fl = fr;
      }
    } else {
      double fl = (k0 >= 1) ? face_val<T>(a, base + (k0 - 1) * s, base + k0 * s, k0 - 1) : 0.0;
      for (int64_t k = k0; k < k1; ++k) {
        const double fr = (k < N) ? face_val<T>(a, base + k * s, base + (k + 1) * s, k) : 0.0;
        const double old = a.accumulate ? (double)static_cast<const T*>(a.acc)[base + k * s] : 0.0;
        const double div = (k == 0 || k == N) ? 0.0 : rn_mul(rn_sub(fr, fl), node_inv_w(a, k));
        static_cast<T*>(a.acc)[base + k * s] = (T)rn_add(old, -div);
        fl = fr;
      }
    }
  }
}

struct Shape3 {
  int64_t n[3];
  int per[3];
  int ndim;
};

// node whose value the periodic image node x takes (every periodic coordinate
// N -> 0, as sync_periodic_image_nodes applies the axes in turn)
__device__ __forceinline__ int64_t image_source(const Shape3& s, int64_t i) {
  int64_t c[3] = {0, 0, 0}, r = i;
  for (int a = s.ndim - 1; a >= 0; --a) {
    c[a] = r % s.n[a];
    r /= s.n[a];
  }
  int64_t j = 0;
  for (int a = 0; a < s.ndim; ++a) {
    const int64_t ca = (s.per[a] && c[a] == s.n[a] - 1) ? 0 : c[a];
    j = j * s.n[a] + ca;
  }
  return j;
}

// TVD-RK3 stage (tvd_rk3.py:26-48) with the post-stage clip and image sync
// (fccd_advection.py:116-120): stage 0: q (clip and sync only); stage 1:
// q + dt L; stages 2, 3:
// a q0 + b (q + dt L); then clip to [lo, hi] (NaN kept) and the periodic
// image nodes take their source node's value.
template <typename T>
__global__ void rk3_stage_kernel(Shape3 s, int stage, double ca, double cb, double dt, const T* q0, const T* q,
                                 const T* L, int clip, double lo, double hi, int any_per, T* out) {
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = any_per ? image_source(s, i) : i;
    double v;
    if (stage == 0) {
      v = (double)q[j];
    } else {
      const double up = rn_add((double)q[j], rn_mul(dt, (double)L[j]));
      v = (stage == 1) ? up : rn_add(rn_mul(ca, (double)q0[j]), rn_mul(cb, up));
    }
    v = (double)(T)v;
    if (clip) v = v < lo ? lo : (v > hi ? hi : v);
    out[i] = (T)v;
  }
}

template <typename T>
__global__ void sync_images_kernel(Shape3 s, T* arr) {
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = image_source(s, i);
    if (j != i) arr[i] = arr[j];   // sources have no coordinate at N: never written
  }
}

int make_shape(int ndim, const int64_t* shape, const int* periodic, Shape3& s) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape, "ndim must be 1..3");
  s.ndim = ndim;
  for (int a = 0; a < 3; ++a) {
    s.n[a] = 1;
    s.per[a] = 0;
  }
  for (int a = 0; a < ndim; ++a) {
    TPF_CHECK_ARG(shape[a] >= 1, "empty axis");
    s.n[a] = shape[a];
    s.per[a] = periodic ? (periodic[a] ? 1 : 0) : 0;
    TPF_CHECK_ARG(!s.per[a] || shape[a] >= 3, "a periodic axis needs at least 3 nodes");
  }
  return TPF_OK;
}

}  // namespace

extern "C" int tpf_fccd_product(int64_t n, const void* u, const void* phi, void* prod, int dtype, void* stream) {
  TPF_CHECK_ARG(n >= 0 && u && phi && prod, "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    product_kernel<double><<<blocks_for(n, 16), 256, 0, st>>>(n, static_cast<const double*>(u),
                                                             static_cast<const double*>(phi), static_cast<double*>(prod));
  else
    product_kernel<float><<<blocks_for(n, 16), 256, 0, st>>>(n, static_cast<const float*>(u),
                                                            static_cast<const float*>(phi), static_cast<float*>(prod));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// the face-value + divergence launch of both entry points below; wf / wn
// NULL on uniform grids (h then gives the constants)
static int flux_divergence_axis(int ndim, const int64_t* shape, int axis, int periodic, double h, const double* wf,
                                const double* wn, const void* prod, const void* q, int accumulate, void* acc,
                                int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape && axis >= 0 && axis < ndim, "invalid shape or axis");
  TPF_CHECK_ARG(prod && q && acc && acc != prod && acc != q, "NULL or aliased argument");
  TPF_CHECK_ARG(h > 0.0, "h must be positive");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  FluxArgs a{};
  a.prod = prod; a.q = q; a.acc = acc;
  a.wf = wf; a.wn = wn;
  a.outer = 1; a.inner = 1;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(shape[d] >= 1, "empty axis");
    if (d < axis) a.outer *= shape[d];
    if (d > axis) a.inner *= shape[d];
  }
  a.n = shape[axis];
  TPF_CHECK_ARG(a.n >= (periodic ? 3 : 2), "too few nodes along the axis (%lld)", (long long)a.n);
  // the reference's constants: inv_H = 1/H, H^2/16 = H*H/16 (fccd_helpers.py:23-34)
  a.inv_h = 1.0 / h;
  a.h2_16 = (h * h) / 16.0;
  a.periodic = periodic ? 1 : 0;
  a.accumulate = accumulate ? 1 : 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t tot = a.outer * a.n * a.inner;
  if (a.inner >= 32) {
    const int64_t lines = a.outer * a.inner, sms = tpf::sm_count();
    // nodes per thread along the axis: autotuned among kChunks (the march
    // gives the same values for every chunk length), else enough threads to
    // fill the GPU (about 2048 per SM), 8..64 nodes
    int64_t chunk = (lines * a.n) / (sms * 2048);
    chunk = std::max<int64_t>(8, std::min<int64_t>(64, chunk));
    static constexpr int64_t kChunks[5] = {8, 16, 32, 64, 128};
    auto launch = [&](int64_t ck, void* out, cudaStream_t s2) -> int {
      FluxArgs b = a;
      b.acc = out;
      const int64_t nchunks = (a.n + ck - 1) / ck;
      const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((lines * nchunks + 255) / 256, sms * 8));
      if (dtype == TPF_F64) flux_march_kernel<double><<<blocks, 256, 0, s2>>>(b, ck, nchunks);
      else flux_march_kernel<float><<<blocks, 256, 0, s2>>>(b, ck, nchunks);
      return cudaPeekAtLastError() == cudaSuccess ? TPF_OK : TPF_ECUDA;
    };
    auto cand = [&](int c, void* scratch, cudaStream_t s2) { return launch(kChunks[c], scratch, s2); };
    const tpf::TuneKey key{tpf::kTuneFluxMarch, dtype,
                           {a.outer, a.n, a.inner, 2 * a.periodic + a.accumulate + (wf ? 4 : 0)}};
    const int pick = tpf::tuned_choice(key, 5, -1, (size_t)tot * (dtype == TPF_F64 ? 8 : 4), st, cand);
    launch(pick >= 0 ? kChunks[pick] : chunk, a.acc, st);
  } else {
    if (dtype == TPF_F64) flux_div_kernel<double><<<blocks_for(tot, 16), 256, 0, st>>>(a);
    else flux_div_kernel<float><<<blocks_for(tot, 16), 256, 0, st>>>(a);
  }
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_fccd_flux_divergence_axis(int ndim, const int64_t* shape, int axis, int periodic, double h,
                                             const void* prod, const void* q, int accumulate, void* acc, int dtype,
                                             void* stream) {
  return flux_divergence_axis(ndim, shape, axis, periodic, h, nullptr, nullptr, prod, q, accumulate, acc, dtype,
                              stream);
}

extern "C" int tpf_fccd_flux_divergence_axis_nonuniform(int ndim, const int64_t* shape, int axis, int periodic,
                                                        const double* face_h2_16, const double* node_inv_width,
                                                        const void* prod, const void* q, int accumulate, void* acc,
                                                        int dtype, void* stream) {
  TPF_CHECK_ARG(face_h2_16 && node_inv_width, "NULL weight array");
  return flux_divergence_axis(ndim, shape, axis, periodic, 1.0, face_h2_16, node_inv_width, prod, q, accumulate, acc,
                              dtype, stream);
}

// Option C node gradient (FCCDSolver.node_gradient, fccd.py:90-94,131-134,
// 243-277,392-462): face gradients d_f = (u_hi - u_lo)/H - (H/24)(q_hi - q_lo)
// and the R_4 Hermite reconstruction 0.5 (d_L + d_R) - (H/16)(q_{i+1} -
// q_{i-1}) at the nodes; wall nodes 0 and N take their one face gradient,
// periodic axes wrap over the N unique nodes and node N repeats node 0.
// mode 0: out = g; 1: out = 0 - uk g (the first term of the nodal advection
// sum, fccd_advection_helpers.py:46-72); 2: out -= uk g.
template <typename T>
__global__ void fccd_node_grad_kernel(int64_t outer, int64_t n, int64_t inner, int periodic, double inv_h, double h24,
                                      double h16, const double* winv, const double* w24, const double* w16,
                                      const T* u, const T* q, const T* uk, int mode, T* out) {
  const int64_t tot = outer * n * inner, N = n - 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t in = i % inner, k = (i / inner) % n, o = i / (inner * n);
    const int64_t base = o * n * inner + in;
    auto at = [&](const T* f, int64_t j) { return (double)f[base + j * inner]; };
    // face gradient between nodes j and j+1 (periodic: j+1 wraps over N unique nodes)
    auto dface = [&](int64_t j) {
      const int64_t jp = periodic ? (j + 1 == N ? 0 : j + 1) : j + 1;
      const double ih = winv ? winv[j] : inv_h, c24 = w24 ? w24[j] : h24;
      return rn_sub(rn_mul(rn_sub(at(u, jp), at(u, j)), ih), rn_mul(c24, rn_sub(at(q, jp), at(q, j))));
    };
    double g;
    if (periodic) {
      const int64_t kk = (k == N) ? 0 : k;
      const int64_t km = (kk == 0) ? N - 1 : kk - 1, kp = (kk + 1 == N) ? 0 : kk + 1;
      g = rn_sub(rn_mul(0.5, rn_add(dface(km), dface(kk))), rn_mul(w16 ? w16[kk] : h16, rn_sub(at(q, kp), at(q, km))));
    } else if (k == 0) {
      g = dface(0);
    } else if (k == N) {
      g = dface(N - 1);
    } else {
      g = rn_sub(rn_mul(0.5, rn_add(dface(k - 1), dface(k))),
                 rn_mul(w16 ? w16[k] : h16, rn_sub(at(q, k + 1), at(q, k - 1))));
    }
    if (mode == 0) {
      out[i] = (T)g;
    } else {
      const double prev = (mode == 1) ? 0.0 : (double)out[i];
      out[i] = (T)rn_sub(prev, rn_mul((double)uk[i], g));
    }
  }
}

static int node_gradient_axis(int ndim, const int64_t* shape, int axis, int periodic, double h, const double* winv,
                              const double* w24, const double* w16, const void* u, const void* q, const void* uk,
                              int mode, void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape && axis >= 0 && axis < ndim, "invalid shape or axis");
  TPF_CHECK_ARG(u && q && out && out != u && out != q && (mode == 0 || (uk && out != uk)), "NULL or aliased argument");
  TPF_CHECK_ARG(mode >= 0 && mode <= 2, "mode must be 0 (gradient), 1 (0 - uk g) or 2 (out -= uk g)");
  TPF_CHECK_ARG(h > 0.0, "h must be positive");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  int64_t outer = 1, inner = 1;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(shape[d] >= 1, "empty axis");
    if (d < axis) outer *= shape[d];
    if (d > axis) inner *= shape[d];
  }
  const int64_t n = shape[axis];
  TPF_CHECK_ARG(n >= (periodic ? 3 : 2), "too few nodes along the axis (%lld)", (long long)n);
  // the reference's constants: 1/H, H/24, H/16 (fccd_helpers.py:23-35)
  const double inv_h = 1.0 / h, h24 = h / 24.0, h16 = h / 16.0;
  const int64_t tot = outer * n * inner;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    fccd_node_grad_kernel<double><<<blocks_for(tot, 16), 256, 0, st>>>(
        outer, n, inner, periodic ? 1 : 0, inv_h, h24, h16, winv, w24, w16, static_cast<const double*>(u),
        static_cast<const double*>(q), static_cast<const double*>(uk), mode, static_cast<double*>(out));
  else
    fccd_node_grad_kernel<float><<<blocks_for(tot, 16), 256, 0, st>>>(
        outer, n, inner, periodic ? 1 : 0, inv_h, h24, h16, winv, w24, w16, static_cast<const float*>(u),
        static_cast<const float*>(q), static_cast<const float*>(uk), mode, static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_fccd_node_gradient_axis(int ndim, const int64_t* shape, int axis, int periodic, double h,
                                           const void* u, const void* q, const void* uk, int mode, void* out,
                                           int dtype, void* stream) {
  return node_gradient_axis(ndim, shape, axis, periodic, h, nullptr, nullptr, nullptr, u, q, uk, mode, out, dtype,
                            stream);
}

extern "C" int tpf_fccd_node_gradient_axis_nonuniform(int ndim, const int64_t* shape, int axis, int periodic,
                                                      const double* face_inv_h, const double* face_h_24,
                                                      const double* node_h_16, const void* u, const void* q,
                                                      const void* uk, int mode, void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(face_inv_h && face_h_24 && node_h_16, "NULL weight array");
  return node_gradient_axis(ndim, shape, axis, periodic, 1.0, face_inv_h, face_h_24, node_h_16, u, q, uk, mode, out,
                            dtype, stream);
}

extern "C" int tpf_tvd_rk3_stage(int ndim, const int64_t* shape, const int* periodic, int stage, double ca, double cb,
                                 double dt, const void* q0, const void* q, const void* L, int clip, double lo,
                                 double hi, void* out, int dtype, void* stream) {
  Shape3 s;
  const int rc = make_shape(ndim, shape, periodic, s);
  if (rc != TPF_OK) return rc;
  TPF_CHECK_ARG(stage >= 0 && stage <= 3, "stage must be 0, 1, 2 or 3");
  TPF_CHECK_ARG(q && out && (stage == 0 || L) && (stage <= 1 || q0), "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  int any_per = 0;
  for (int a = 0; a < ndim; ++a) any_per |= s.per[a];
  // out may equal q or L only without periodic axes (the image nodes read
  // their source nodes, which another thread may already have overwritten)
  TPF_CHECK_ARG(!any_per || (out != q && (stage == 0 || out != L) && (stage <= 1 || out != q0)),
                "with periodic axes the stage output must not alias its inputs");
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    rk3_stage_kernel<double><<<blocks_for(tot, 16), 256, 0, st>>>(
        s, stage, ca, cb, dt, static_cast<const double*>(q0), static_cast<const double*>(q),
        static_cast<const double*>(L), clip, lo, hi, any_per, static_cast<double*>(out));
  else
    rk3_stage_kernel<float><<<blocks_for(tot, 16), 256, 0, st>>>(
        s, stage, ca, cb, dt, static_cast<const float*>(q0), static_cast<const float*>(q),
        static_cast<const float*>(L), clip, lo, hi, any_per, static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_sync_periodic_images(int ndim, const int64_t* shape, const int* periodic, void* arr, int dtype,
                                        void* stream) {
  Shape3 s;
  const int rc = make_shape(ndim, shape, periodic, s);
  if (rc != TPF_OK) return rc;
  TPF_CHECK_ARG(arr, "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  int any_per = 0;
  for (int a = 0; a < ndim; ++a) any_per |= s.per[a];
  if (!any_per) return TPF_OK;
  const int64_t tot = s.n[0] * s.n[1] * s.n[2];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64) sync_images_kernel<double><<<blocks_for(tot, 16), 256, 0, st>>>(s, static_cast<double*>(arr));
  else sync_images_kernel<float><<<blocks_for(tot, 16), 256, 0, st>>>(s, static_cast<float*>(arr));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// ---------------------------------------------------------------------------
// Split reinitialization (levelset/reinit_split.py:73-102, reinit_ops.py:54-204,
// heaviside.py:118-149): compression flux psi(1-psi) n, its filtered CCD
// divergence, the CN-ADI line solves and the interface-weighted mass
// correction.
// ---------------------------------------------------------------------------
namespace {

struct CompArgs {
  const void* d1[3];
  void* flux[3];
  const void* psi;
  int64_t n;
  int ndim;
};

// flux_a = psi (1 - psi) * d1_a / max(sqrt(max(|grad psi|^2, 1e-12)), 1e-6)
// (compute_gradient_normal, reinit_ops.py:57-80, and dccd_compression_div :108-114)
template <typename T>
__global__ void compression_flux_kernel(CompArgs a) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x) {
    double g[3] = {0.0, 0.0, 0.0};
    double gs = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < a.ndim) {
        g[d] = (double)static_cast<const T*>(a.d1[d])[i];
        gs = rn_add(gs, rn_mul(g[d], g[d]));
      }
    double sg = sqrt(gs > 1e-12 || gs != gs ? gs : 1e-12);
    sg = (sg > 1e-6 || sg != sg) ? sg : 1e-6;
    const double p = (double)static_cast<const T*>(a.psi)[i];
    const double pp = rn_mul(p, rn_sub(1.0, p));
#pragma unroll
    for (int d = 0; d < 3; ++d)
      if (d < a.ndim) static_cast<T*>(a.flux[d])[i] = (T)rn_mul(pp, g[d] / sg);
  }
}

// div (+)= g[c] + eps_d ((g[c+1] - 2 g[c]) + g[c-1]) along one axis, the ends
// padded by one ghost node: 0 ('zero'), the opposite interior node
// ('periodic': g[n-2] left, g[1] right) or the end node itself ('neumann',
// 'outflow') (filtered_divergence, reinit_ops.py:83-105; pad_ghost_cells,
// core/boundary.py:249-292).
template <typename T>
__global__ void filtered_div_kernel(int64_t outer, int64_t n, int64_t inner, int pad, double eps_d, const T* g,
                                    const double* J, int accumulate, T* div) {
  const int64_t tot = outer * n * inner;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = (i / inner) % n;
    const double c = (double)g[i];
    double m, p;
    if (k > 0) m = (double)g[i - inner];
    else m = pad == 0 ? 0.0 : (pad == 1 ? (double)g[i + (n - 2) * inner] : c);
    if (k < n - 1) p = (double)g[i + inner];
    else p = pad == 0 ? 0.0 : (pad == 1 ? (double)g[i - (n - 2) * inner] : c);
    double v = rn_add(c, rn_mul(eps_d, rn_add(rn_sub(p, rn_mul(2.0, c)), m)));
    if (J) v = rn_mul(J[k], v);   // non-uniform: the filter in xi-space, then J (reinit_ops.py:95-105)
    div[i] = (T)(accumulate ? rn_add((double)div[i], v) : rn_add(0.0, v));
  }
}

// CN half-step along one axis (cn_diffusion_axis, reinit_ops.py:169-204):
// rhs = (M2 + mu B2) psi with the mirrored end rows, then the Thomas sweep
// with the factors f, m, sup built once on the host (build_cn_factors).
// One thread per line, consecutive threads on consecutive lines.  Both sweeps
// fetch CN_CHUNK nodes ahead into registers before the dependent arithmetic,
// so a line's loads overlap instead of each step waiting for one (a 2-D grid
// has only N+1 lines, one thread each).
constexpr int CN_CHUNK = 8;

template <typename T>
__global__ void __launch_bounds__(256) cn_line_kernel(int64_t outer, int64_t n, int64_t inner, double cR, double dR,
                                                      const double* f, const double* m, const double* sup,
                                                      const T* in, T* out) {
  const int64_t lines = outer * inner;
  const double c2 = rn_mul(2.0, cR);
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < lines; l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = l / inner, in_ = l - o * inner;
    const int64_t base = o * n * inner + in_;
    // forward: node k's rhs needs psi at k-1, k, k+1; d stored in out
    double pm = 0.0, pc = (double)in[base];
    double d = 0.0;
    for (int64_t k0 = 0; k0 < n; k0 += CN_CHUNK) {
      double nx[CN_CHUNK];   // psi at k+1 for k = k0 .. k0+CN_CHUNK-1
#pragma unroll
      for (int j = 0; j < CN_CHUNK; ++j) {
        const int64_t k = k0 + j + 1;
        nx[j] = k < n ? (double)in[base + k * inner] : 0.0;
      }
      double fk[CN_CHUNK];
#pragma unroll
      for (int j = 0; j < CN_CHUNK; ++j) {
        const int64_t k = k0 + j;
        fk[j] = (k >= 1 && k < n) ? f[k - 1] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < CN_CHUNK; ++j) {
        const int64_t k = k0 + j;
        if (k >= n) break;
        const double pn = nx[j];
        double r;
        if (k == 0) r = rn_add(rn_mul(dR, pc), rn_mul(c2, pn));
        else if (k < n - 1) r = rn_add(rn_add(rn_mul(cR, pm), rn_mul(dR, pc)), rn_mul(cR, pn));
        else r = rn_add(rn_mul(c2, pm), rn_mul(dR, pc));
        d = (k == 0) ? r : rn_sub(r, rn_mul(fk[j], d));
        out[base + k * inner] = (T)d;
        pm = pc;
        pc = pn;
      }
    }
    // back substitution from node n-1 down, CN_CHUNK stored d values at a time
    double x = d / m[n - 1];
    out[base + (n - 1) * inner] = (T)x;
    for (int64_t k1 = n - 2; k1 >= 0; k1 -= CN_CHUNK) {
      double dk[CN_CHUNK], sk[CN_CHUNK], mk[CN_CHUNK];
#pragma unroll
      for (int j = 0; j < CN_CHUNK; ++j) {
        const int64_t k = k1 - j;
        dk[j] = k >= 0 ? (double)out[base + k * inner] : 0.0;
        sk[j] = k >= 0 ? sup[k] : 0.0;
        mk[j] = k >= 0 ? m[k] : 1.0;
      }
#pragma unroll
      for (int j = 0; j < CN_CHUNK; ++j) {
        const int64_t k = k1 - j;
        if (k < 0) break;
        x = rn_sub(dk[j], rn_mul(sk[j], x)) / mk[j];
        out[base + k * inner] = (T)x;
      }
    }
  }
}

// The same CN half-step on the contiguous axis (inner == 1).  There the 32
// lines of a warp's group are consecutive in memory, so a chunk of CNC_KC
// nodes of all 32 lines is staged through shared memory with one coalesced
// 256-byte access per line (lane = node), and lane l runs line l's recurrences
// from the tile: the forward sweep over the staged psi (d written back through
// the tile, coalesced), then the back substitution over the staged d -- the
// arithmetic of cn_line_kernel in the same order, so the results are the
// same bits.  (One thread per line reading its own contiguous line touches a
// different 32-byte sector per lane on every load.)
constexpr int CNC_KC = 32;
constexpr int CNC_WARPS = 4;

template <typename T>
__global__ void __launch_bounds__(CNC_WARPS * 32) cn_contig_kernel(int64_t lines, int64_t n, double cR, double dR,
                                                                   const double* f, const double* m,
                                                                   const double* sup, const T* in, T* out) {
  __shared__ double tile_all[CNC_WARPS][32][CNC_KC + 1];
  __shared__ double coef_all[CNC_WARPS][2][CNC_KC];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double(*tile)[CNC_KC + 1] = tile_all[wid];
  double* ca = coef_all[wid][0];
  double* cb = coef_all[wid][1];
  const double c2 = rn_mul(2.0, cR);
  const int64_t ngroups = (lines + 31) / 32;
  for (int64_t g = blockIdx.x * (int64_t)CNC_WARPS + wid; g < ngroups; g += (int64_t)gridDim.x * CNC_WARPS) {
    const int64_t l0 = g * 32;
    const int nl = (int)(lines - l0 < 32 ? lines - l0 : 32);
    const T* gin = in + l0 * n;   // line j of the group starts at gin + j n
    T* gout = out + l0 * n;
    const bool act = lane < nl;
    double pm = 0.0, pc = act ? (double)gin[(int64_t)lane * n] : 0.0;
    double d = 0.0;
    // forward sweep, chunks of nodes k0 .. k0 + cnt - 1
    for (int64_t k0 = 0; k0 < n; k0 += CNC_KC) {
      const int cnt = (int)(n - k0 < CNC_KC ? n - k0 : CNC_KC);
      {
        const int64_t k = k0 + 1 + lane;   // psi at k + 1 for the chunk's nodes
        double v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = (j < nl && k < n) ? (double)gin[(int64_t)j * n + k] : 0.0;
#pragma unroll
        for (int j = 0; j < 32; ++j) tile[j][lane] = v[j];
        const int64_t kc = k0 + lane;
        ca[lane] = (kc >= 1 && kc < n) ? f[kc - 1] : 0.0;
      }
      __syncwarp();
      for (int t = 0; t < cnt; ++t) {
        const int64_t k = k0 + t;
        const double pn = tile[lane][t];
        double r;
        if (k == 0) r = rn_add(rn_mul(dR, pc), rn_mul(c2, pn));
        else if (k < n - 1) r = rn_add(rn_add(rn_mul(cR, pm), rn_mul(dR, pc)), rn_mul(cR, pn));
        else r = rn_add(rn_mul(c2, pm), rn_mul(dR, pc));
        d = (k == 0) ? r : rn_sub(r, rn_mul(ca[t], d));
        tile[lane][t] = d;
        pm = pc;
        pc = pn;
      }
      __syncwarp();
      if (lane < cnt) {
        for (int j = 0; j < nl; ++j) gout[(int64_t)j * n + k0 + lane] = (T)tile[j][lane];
      }
      __syncwarp();
    }
    // back substitution: node n - 1 from the unrounded d, then down from n - 2
    // over the stored (T-rounded) d, chunks of nodes kb .. kb + cnt - 1 from the top
    double x = d / m[n - 1];
    for (int64_t top = n - 1; top >= 0; top -= CNC_KC) {
      const int64_t kb = top - CNC_KC + 1 > 0 ? top - CNC_KC + 1 : 0;
      const int cnt = (int)(top - kb + 1);
      if (lane < cnt) {
        for (int j = 0; j < nl; ++j) tile[j][lane] = (double)gout[(int64_t)j * n + kb + lane];
        ca[lane] = sup[kb + lane < n - 1 ? kb + lane : 0];
        cb[lane] = m[kb + lane];
      }
      __syncwarp();
      for (int t = cnt - 1; t >= 0; --t) {
        const int64_t k = kb + t;
        if (k < n - 1) x = rn_sub(tile[lane][t], rn_mul(ca[t], x)) / cb[t];
        tile[lane][t] = x;
      }
      __syncwarp();
      if (lane < cnt) {
        for (int j = 0; j < nl; ++j) gout[(int64_t)j * n + kb + lane] = (T)tile[j][lane];
      }
      __syncwarp();
    }
  }
}

constexpr int MASS_BLOCKS = 1024;

// per-block partial sums of q dV and 4 q (1 - q) dV in a fixed order
template <typename T>
__global__ void mass_partials_kernel(int64_t n, const T* q, const double* dV, double* part) {
  __shared__ double s0[256], s1[256];
  double a0 = 0.0, a1 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double qi = (double)q[i], dv = dV[i];
    a0 = rn_add(a0, rn_mul(qi, dv));
    a1 = rn_add(a1, rn_mul(rn_mul(rn_mul(4.0, qi), rn_sub(1.0, qi)), dv));
  }
  s0[threadIdx.x] = a0;
  s1[threadIdx.x] = a1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] = rn_add(s0[threadIdx.x], s0[threadIdx.x + w]);
      s1[threadIdx.x] = rn_add(s1[threadIdx.x], s1[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s0[0];
    part[MASS_BLOCKS + blockIdx.x] = s1[0];
  }
}

// sums[0] = sum q dV, sums[1] = sum w dV from the partials (one block, fixed order)
__global__ void mass_finish_kernel(int nb, const double* part, double* sums) {
  __shared__ double s0[256], s1[256];
  double a0 = 0.0, a1 = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    a0 = rn_add(a0, part[i]);
    a1 = rn_add(a1, part[MASS_BLOCKS + i]);
  }
  s0[threadIdx.x] = a0;
  s1[threadIdx.x] = a1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] = rn_add(s0[threadIdx.x], s0[threadIdx.x + w]);
      s1[threadIdx.x] = rn_add(s1[threadIdx.x], s1[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[0] = s0[0];
    sums[1] = s1[0];
  }
}

// q <- clip(q + gate (M_target - M_new) / W_safe * w, 0, 1) (apply_mass_correction)
template <typename T>
__global__ void mass_apply_kernel(int64_t n, const T* q, const double* target, const double* sums, T* out) {
  const double W = sums[1];
  const double Ws = W > 1e-12 ? W : 1.0;
  const double ratio = rn_sub(target[0], sums[0]) / Ws;
  const double gr = rn_mul(W > 1e-12 ? 1.0 : 0.0, ratio);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double qi = (double)q[i];
    const double w = rn_mul(rn_mul(4.0, qi), rn_sub(1.0, qi));
    double v = rn_add(qi, rn_mul(gr, w));
    v = (double)(T)v;
    v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    out[i] = (T)v;
  }
}

}  // namespace

extern "C" int tpf_reinit_compression_flux(int ndim, int64_t n, const void* psi, const void* const* d1,
                                           void* const* flux, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && n >= 0 && psi && d1 && flux, "invalid arguments");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  CompArgs a{};
  a.psi = psi; a.n = n; a.ndim = ndim;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(d1[d] && flux[d], "NULL derivative or flux %d", d);
    a.d1[d] = d1[d];
    a.flux[d] = flux[d];
  }
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64) compression_flux_kernel<double><<<blocks_for(n, 16), 256, 0, st>>>(a);
  else compression_flux_kernel<float><<<blocks_for(n, 16), 256, 0, st>>>(a);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

static int filtered_divergence_axis(int ndim, const int64_t* shape, int axis, int pad, double eps_d, const double* J,
                                    const void* g, int accumulate, void* div, int dtype, void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape && axis >= 0 && axis < ndim, "invalid shape or axis");
  TPF_CHECK_ARG(pad >= 0 && pad <= 2, "pad must be 0 (zero), 1 (periodic) or 2 (neumann/outflow)");
  TPF_CHECK_ARG(g && div && g != div, "NULL or aliased argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  int64_t outer = 1, inner = 1;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(shape[d] >= 1, "empty axis");
    if (d < axis) outer *= shape[d];
    if (d > axis) inner *= shape[d];
  }
  const int64_t n = shape[axis];
  TPF_CHECK_ARG(n >= 3, "at least 3 nodes along the axis");
  const int64_t tot = outer * n * inner;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    filtered_div_kernel<double><<<blocks_for(tot, 16), 256, 0, st>>>(outer, n, inner, pad, eps_d,
                                                                    static_cast<const double*>(g), J, accumulate,
                                                                    static_cast<double*>(div));
  else
    filtered_div_kernel<float><<<blocks_for(tot, 16), 256, 0, st>>>(outer, n, inner, pad, eps_d,
                                                                   static_cast<const float*>(g), J, accumulate,
                                                                   static_cast<float*>(div));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_reinit_filtered_divergence_axis(int ndim, const int64_t* shape, int axis, int pad, double eps_d,
                                                   const void* g, int accumulate, void* div, int dtype,
                                                   void* stream) {
  return filtered_divergence_axis(ndim, shape, axis, pad, eps_d, nullptr, g, accumulate, div, dtype, stream);
}

extern "C" int tpf_reinit_filtered_divergence_axis_metric(int ndim, const int64_t* shape, int axis, int pad,
                                                          double eps_d, const double* J, const void* g,
                                                          int accumulate, void* div, int dtype, void* stream) {
  TPF_CHECK_ARG(J, "NULL metric");
  return filtered_divergence_axis(ndim, shape, axis, pad, eps_d, J, g, accumulate, div, dtype, stream);
}

extern "C" int tpf_reinit_cn_axis(int ndim, const int64_t* shape, int axis, double cR, double dR, const double* f,
                                  const double* m, const double* sup, const void* in, void* out, int dtype,
                                  void* stream) {
  TPF_CHECK_ARG(ndim >= 1 && ndim <= 3 && shape && axis >= 0 && axis < ndim, "invalid shape or axis");
  TPF_CHECK_ARG(f && m && sup && in && out && in != out, "NULL or aliased argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  int64_t outer = 1, inner = 1;
  for (int d = 0; d < ndim; ++d) {
    TPF_CHECK_ARG(shape[d] >= 1, "empty axis");
    if (d < axis) outer *= shape[d];
    if (d > axis) inner *= shape[d];
  }
  const int64_t n = shape[axis];
  TPF_CHECK_ARG(n >= 2, "at least 2 nodes along the axis");
  const int64_t lines = outer * inner;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (inner == 1) {
    // contiguous axis: groups of 32 consecutive lines staged through shared memory
    const int64_t ngroups = (lines + 31) / 32;
    const int blocks = (int)std::max<int64_t>(
        1, std::min<int64_t>((ngroups + CNC_WARPS - 1) / CNC_WARPS, (int64_t)tpf::sm_count() * 8));
    if (dtype == TPF_F64)
      cn_contig_kernel<double><<<blocks, CNC_WARPS * 32, 0, st>>>(lines, n, cR, dR, f, m, sup,
                                                                  static_cast<const double*>(in),
                                                                  static_cast<double*>(out));
    else
      cn_contig_kernel<float><<<blocks, CNC_WARPS * 32, 0, st>>>(lines, n, cR, dR, f, m, sup,
                                                                 static_cast<const float*>(in),
                                                                 static_cast<float*>(out));
    TPF_CUDA_TRY(cudaGetLastError());
    return TPF_OK;
  }
  // one thread per line; threads per block autotuned among kThreadsCand (a
  // line's solve does not depend on the launch shape), else 256 with up to
  // 8 blocks per SM
  static constexpr int kThreadsCand[3] = {64, 128, 256};
  const int64_t sms = tpf::sm_count();
  auto launch = [&](int bs, void* dst, cudaStream_t s2) -> int {
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((lines + bs - 1) / bs, sms * (2048 / bs)));
    if (dtype == TPF_F64)
      cn_line_kernel<double><<<blocks, bs, 0, s2>>>(outer, n, inner, cR, dR, f, m, sup, static_cast<const double*>(in),
                                                    static_cast<double*>(dst));
    else
      cn_line_kernel<float><<<blocks, bs, 0, s2>>>(outer, n, inner, cR, dR, f, m, sup, static_cast<const float*>(in),
                                                   static_cast<float*>(dst));
    return cudaPeekAtLastError() == cudaSuccess ? TPF_OK : TPF_ECUDA;
  };
  auto cand = [&](int c, void* scratch, cudaStream_t s2) { return launch(kThreadsCand[c], scratch, s2); };
  const tpf::TuneKey key{tpf::kTuneCnLine, dtype, {outer, n, inner, 0}};
  const int pick = tpf::tuned_choice(key, 3, -1, (size_t)(outer * n * inner) * (dtype == TPF_F64 ? 8 : 4), st, cand);
  if (pick >= 0) {
    launch(kThreadsCand[pick], out, st);
  } else if (dtype == TPF_F64) {
    cn_line_kernel<double><<<blocks_for(lines, 8), 256, 0, st>>>(outer, n, inner, cR, dR, f, m, sup,
                                                                 static_cast<const double*>(in),
                                                                 static_cast<double*>(out));
  } else {
    cn_line_kernel<float><<<blocks_for(lines, 8), 256, 0, st>>>(outer, n, inner, cR, dR, f, m, sup,
                                                                static_cast<const float*>(in),
                                                                static_cast<float*>(out));
  }
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_mass_sums(int64_t n, const void* q, const double* dV, double* partials, double* sums, int dtype,
                             void* stream) {
  TPF_CHECK_ARG(n >= 1 && q && dV && partials && sums, "invalid arguments");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = (int)std::min<int64_t>(MASS_BLOCKS, (n + 255) / 256);
  if (dtype == TPF_F64) mass_partials_kernel<double><<<nb, 256, 0, st>>>(n, static_cast<const double*>(q), dV, partials);
  else mass_partials_kernel<float><<<nb, 256, 0, st>>>(n, static_cast<const float*>(q), dV, partials);
  mass_finish_kernel<<<1, 256, 0, st>>>(nb, partials, sums);
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

extern "C" int tpf_mass_correction_apply(int64_t n, const void* q, const double* target, const double* sums,
                                         void* out, int dtype, void* stream) {
  TPF_CHECK_ARG(n >= 1 && q && target && sums && out, "invalid arguments");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    mass_apply_kernel<double><<<blocks_for(n, 16), 256, 0, st>>>(n, static_cast<const double*>(q), target, sums,
                                                                 static_cast<double*>(out));
  else
    mass_apply_kernel<float><<<blocks_for(n, 16), 256, 0, st>>>(n, static_cast<const float*>(q), target, sums,
                                                                static_cast<float*>(out));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

// ---------------------------------------------------------------------------
// UCCD6 convection accumulation (UCCD6ConvectionTerm.compute,
// src/twophase/ns_terms/uccd6_convection.py:83-128), per (component j, axis k):
//   acc = acc - 0.5 (u_k d1 + dcons);  acc = acc - coeff (u_ref d8)
// with d1 = D1_k u_j, dcons = D1_k (u_k u_j), d8 = (D2_k)^4 u_j from the CCD
// kernels, u_ref = max |u_k| (device scalar), coeff = sigma h_k^7.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void uccd6_acc_kernel(int64_t n, int first, const T* uk, const T* d1, const T* cons, const T* d8,
                                 double coeff, const double* uref, T* acc) {
  const double ur = *uref;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double a0 = first ? 0.0 : (double)acc[i];
    const double adv = rn_mul((double)uk[i], (double)d1[i]);
    double a = rn_sub(a0, rn_mul(0.5, rn_add(adv, (double)cons[i])));
    a = (double)(T)a;
    a = rn_sub(a, rn_mul(coeff, rn_mul(ur, (double)d8[i])));
    acc[i] = (T)a;
  }
}

}  // namespace

extern "C" int tpf_uccd6_accumulate(int64_t n, int first, const void* uk, const void* d1, const void* cons,
                                    const void* d8, double coeff, const double* uref, void* acc, int dtype,
                                    void* stream) {
  TPF_CHECK_ARG(n >= 0 && uk && d1 && cons && d8 && uref && acc, "NULL argument");
  TPF_CHECK_ARG(dtype == TPF_F64 || dtype == TPF_F32, "dtype must be TPF_F64 or TPF_F32");
  if (n == 0) return TPF_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == TPF_F64)
    uccd6_acc_kernel<double><<<blocks_for(n, 16), 256, 0, st>>>(
        n, first, static_cast<const double*>(uk), static_cast<const double*>(d1), static_cast<const double*>(cons),
        static_cast<const double*>(d8), coeff, uref, static_cast<double*>(acc));
  else
    uccd6_acc_kernel<float><<<blocks_for(n, 16), 256, 0, st>>>(
        n, first, static_cast<const float*>(uk), static_cast<const float*>(d1), static_cast<const float*>(cons),
        static_cast<const float*>(d8), coeff, uref, static_cast<float*>(acc));
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

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

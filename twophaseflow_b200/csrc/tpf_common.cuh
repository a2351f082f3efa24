// Shared helpers of the tpf CUDA library: status codes, error string,
// CUDA error checks, warp/block reductions and a bounded grid barrier.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <string>
#include <utility>

#include "../../include/tpf.h"

namespace tpf {

// Thread-local last-error message returned by tpf_last_error().
void set_error(const char* fmt, ...);
const char* last_error();

#define TPF_CUDA_TRY(expr)                                                     \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      ::tpf::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                       __FILE__, __LINE__);                                    \
      return TPF_ECUDA;                                                        \
    }                                                                          \
  } while (0)

#define TPF_CHECK_ARG(cond, ...)      \
  do {                                \
    if (!(cond)) {                    \
      ::tpf::set_error(__VA_ARGS__);  \
      return TPF_EINVAL;              \
    }                                 \
  } while (0)

// Launch-shape autotuning for kernels whose results do not depend on the
// launch shape (march chunk lengths, threads per block): tuned_choice returns
// the index of the fastest of `ncand` candidates for the signature `key`.
// The first eager call of a signature allocates `scratch_bytes` of zeroed
// scratch, runs each candidate through run(c, scratch, stream) once to warm
// up and three times under CUDA events on `stream`, keeps the fastest for the
// process and frees the scratch; `run` must write only to the scratch.
// Under stream capture, with tuning switched off (tpf_set_launch_autotune),
// or when the scratch cannot be allocated, an untuned signature gets
// `fallback` and nothing is cached.
struct TuneKey {
  int kernel, dtype;
  int64_t d[4];
};
enum TuneKernel { kTuneFluxMarch = 1, kTuneRcMarch = 2, kTuneCnLine = 3 };
typedef int (*TuneRun)(int cand, void* scratch, cudaStream_t s, void* ctx);
int tuned_choice_impl(const TuneKey& key, int ncand, int fallback, size_t scratch_bytes, cudaStream_t s, TuneRun run,
                      void* ctx);
template <typename F>
int tuned_choice(const TuneKey& key, int ncand, int fallback, size_t scratch_bytes, cudaStream_t s, F& f) {
  TuneRun thunk = [](int c, void* scratch, cudaStream_t st, void* ctx) -> int {
    return (*static_cast<F*>(ctx))(c, scratch, st);
  };
  return tuned_choice_impl(key, ncand, fallback, scratch_bytes, s, thunk, &f);
}

inline int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 1;
}

// ---- programmatic dependent launch for chains of short dependent kernels ----
// A kernel launched by launch_chained may be launched (its launch and block
// scheduling overlapping the previous kernel's tail) before its predecessor in
// the stream has finished; it must call chain_begin() before it touches any
// memory: that waits until the predecessor has completed with its memory
// visible.  chain_end(), the last statement of a chained kernel, lets the next
// kernel launch once every block has reached it (blocks that return early
// count when they exit).  Without the launch attribute (plain <<< >>>
// launches) both return at once.
__device__ __forceinline__ void chain_begin() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void chain_end() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                  Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV values; every thread receives the totals.
// scratch must hold NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) scratch[k * 32 + wid] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = (lane < nw) ? scratch[k * 32 + lane] : 0.0;
    v[k] = warp_sum(s);
  }
  __syncthreads();
}

// Grid barrier for cooperatively launched persistent kernels.  Every spin is
// bounded: after `spin_limit` polls the barrier records a timeout in *err and
// returns false so the kernel can leave its loop.  bar[0] = arrival counter,
// bar[1] = generation.
struct GridBarrier {
  unsigned int* bar;
  int* err;
  long long spin_limit;

  __device__ __forceinline__ bool sync(unsigned int nblocks) {
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) {
      volatile unsigned int* vgen = bar + 1;
      unsigned int gen = *vgen;
      __threadfence();
      unsigned int arrived = atomicAdd(bar, 1u);
      if (arrived == nblocks - 1) {
        atomicExch(bar, 0u);
        __threadfence();
        atomicAdd(bar + 1, 1u);
      } else {
        long long spins = 0;
        while (*vgen == gen) {
          if (++spins > spin_limit) {
            atomicExch(err, 1);
            ok = false;
            break;
          }
          if (*(volatile int*)err) { ok = false; break; }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
    __syncthreads();
    // broadcast failure to the whole block
    __shared__ int s_fail;
    if (threadIdx.x == 0) s_fail = ok ? 0 : 1;
    __syncthreads();
    ok = (s_fail == 0);
    __syncthreads();
    return ok;
  }
};

}  // namespace tpf

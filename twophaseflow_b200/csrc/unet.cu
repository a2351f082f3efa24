// Learned pressure-Poisson preconditioner network: a 4-level U-Net
// (3x3 convolutions, channels 16-32-64-128) with BF16 weights and activations
// and FP32 accumulation on the sm_100a tensor cores (tcgen05.mma, accumulators
// in TMEM).  Forward pass for inference and training, backward pass (data
// and weight gradients), Adam.
//
// The reference has no learned component (its PPE is SciPy CG/GMRES), so the
// network is this library's own design:
//
//   encoder  e0 = R(c1(R(c0(x))))            level 0  16 ch   (x = [r~, c~, a~0, a~1])
//            e1 = R(c3(R(c2(pool e0))))      level 1  32 ch
//            e2 = R(c5(R(c4(pool e1))))      level 2  64 ch
//            e3 = R(c7(R(c6(pool e2))))      level 3 128 ch
//   decoder  d2 = R(c9 (R(up(c8 (e3)) + e2)))   level 2
//            d1 = R(c11(R(up(c10(d2)) + e1)))   level 1
//            d0 = R(c13(R(up(c12(d1)) + e0)))   level 0
//   output   y  = 1x1 conv of d0 (16 -> 1)
//
// R = ReLU, pool = 2x2 average, up = 2x nearest.  Decoder convolutions that
// reduce channels run at the coarse level before upsampling.
//
// Activation layout ("stacked padded NHWC"): a batch of B images of level l
// (H_l x W_l, H_l = H >> l) is stored as B consecutive (H_l + 2) x (W_l + 2)
// pixel arrays with a one-pixel zero border, channels innermost.  A 3x3
// convolution is then a uniform shift of the flat pixel index per tap
// (q + dy*Wp + dx), so one 128-pixel tile of outputs needs three 130-pixel
// input windows and every tap's A operand is the same shared-memory window
// at a 16-byte offset -- no im2col copy.  Border outputs are written as zero.
#include "tpf_common.cuh"
#include "tc_sm100.cuh"
#include "ppe_view.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

typedef __nv_bfloat16 bf16;

struct tpf_unet;

namespace {

constexpr int kConvs = 14;
struct LayerSpec {
  int cin, cout, level, relu;
};
// cin of layer 0 is the 4 logical input channels; its kernel input is padded to 16
constexpr int kIn = 4;
constexpr LayerSpec kLayers[kConvs] = {{4, 16, 0, 1},   {16, 16, 0, 1},  {16, 32, 1, 1}, {32, 32, 1, 1},
                                       {32, 64, 2, 1},  {64, 64, 2, 1},  {64, 128, 3, 1}, {128, 128, 3, 1},
                                       {128, 64, 3, 0}, {64, 64, 2, 1},  {64, 32, 2, 0}, {32, 32, 1, 1},
                                       {32, 16, 1, 0},  {16, 16, 0, 1}};
constexpr int kInPad = 16;
constexpr int kOutC = 16;  // channels of d0
constexpr long long kSpin = 1LL << 22;

inline int cin_kernel(int l) { return l == 0 ? kInPad : kLayers[l].cin; }

// flat parameter layout: per layer W[cout][cin][3][3], b[cout]; then w_out[16], b_out
struct ParamLayout {
  int64_t w[kConvs], b[kConvs], wo, bo, total;
  ParamLayout() {
    int64_t o = 0;
    for (int l = 0; l < kConvs; ++l) {
      w[l] = o;
      o += (int64_t)kLayers[l].cout * kLayers[l].cin * 9;
      b[l] = o;
      o += kLayers[l].cout;
    }
    wo = o;
    o += kOutC;
    bo = o;
    o += 1;
    total = o;
  }
};
const ParamLayout& layout() {
  static ParamLayout L;
  return L;
}

// ---- conv geometry shared by host and device -----------------------------------------
constexpr int kTile = 128;           // output pixels per CTA (MMA M)
constexpr int kWin = kTile + 2;      // pixels per input window
constexpr int kPlane = kWin * 16;    // bytes of one 8-channel plane of a window

__host__ __device__ constexpr int taps_per_group(int cin, int cout) {
  return (9 * cin * cout * 2 <= 80 * 1024) ? 9 : 3;
}
__host__ __device__ constexpr int conv_smem_bytes(int cin, int cout) {
  return 3 * (cin / 8) * kPlane + taps_per_group(cin, cout) * cin * cout * 2;
}

struct ConvArgs {
  const bf16* in;     // [P][CIN]
  bf16* out;          // [P][COUT]
  const bf16* w;      // [9][CIN/8][COUT][8]
  const float* bias;  // [COUT] or null
  const bf16* mask;   // [P][COUT] or null: out *= (mask > 0)
  long long P;        // pixels of the stacked padded batch
  int Hp, Wp;         // padded image size
  int relu;
  int* err;
};

__device__ __forceinline__ bool interior_pixel(long long q, int Hp, int Wp) {
  const long long img = (long long)Hp * Wp;
  const int local = (int)(q % img);
  const int yy = local / Wp, xx = local - (local / Wp) * Wp;
  return yy >= 1 && yy <= Hp - 2 && xx >= 1 && xx <= Wp - 2;
}

// One 128-pixel tile of a 3x3 convolution as an implicit GEMM on tcgen05:
// D[pixel][co] = sum_{tap, ci} X[pixel + shift(tap)][ci] * W[tap][co][ci].
// 4 warps; thread 0 issues the MMAs, all warps run the TMEM epilogue.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3x3_tc_kernel(ConvArgs a) {
  using namespace tpf::tc;
  constexpr int KCH = CIN / 8;                 // 16-byte chunks per pixel
  constexpr int WIN_BYTES = KCH * kPlane;
  constexpr int TAP_W = CIN * COUT * 2;        // bytes of one tap's weights
  constexpr int TG = taps_per_group(CIN, COUT);
  constexpr int NCOLS = COUT < 32 ? 32 : COUT;
  constexpr uint32_t IDESC = idesc_bf16_f32(kTile, COUT);
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "conv shape");

  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + 3 * WIN_BYTES;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long q0 = (long long)blockIdx.x * kTile;

  pdl_trigger();   // the next layer may start its prologue
  if (warp == 0) tmem_alloc(&tmem_slot, NCOLS);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_fence_init();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;

  // the first tap group's weights do not depend on the previous layer: load
  // them before waiting for it
  {
    const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
    for (int i = tid; i < TG * TAP_W / 16; i += 128) cp_async16(sB + i * 16, wsrc + i * 16, true);
    cp_async_commit();
  }
  pdl_wait();

  // three input windows (rows dy = -1, 0, +1), 130 pixels each, channel-plane layout
  for (int i = tid; i < 3 * kWin * KCH; i += 128) {
    const int w = i / (kWin * KCH);
    const int rem = i - w * (kWin * KCH);
    const int j = rem / KCH, c = rem - j * KCH;
    const long long q = q0 - 1 + (long long)(w - 1) * a.Wp + j;
    const bool valid = (q >= 0 && q < a.P);
    const bf16* src = a.in + (valid ? q : 0) * CIN + c * 8;
    cp_async16(sA + w * WIN_BYTES + c * kPlane + j * 16, src, valid);
  }
  cp_async_commit();

  bool ok = true;
  uint32_t phase = 0;
  for (int t0 = 0; t0 < 9; t0 += TG) {
    if (t0 > 0) {
      const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w) + (size_t)t0 * TAP_W;
      for (int i = tid; i < TG * TAP_W / 16; i += 128) cp_async16(sB + i * 16, wsrc + i * 16, true);
      cp_async_commit();
    }
    cp_async_wait_all();
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll 1
      for (int tt = 0; tt < TG; ++tt) {
        const int tap = t0 + tt;
        const int dy = tap / 3, dx = tap - (tap / 3) * 3;   // 0..2
        const uint32_t abase = a0 + dy * WIN_BYTES + dx * 16;
        const uint32_t bbase = b0 + tt * TAP_W;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; ++kc) {
          const uint64_t ad = smem_desc(abase + kc * 2 * kPlane, kPlane, 128);
          const uint64_t bd = smem_desc(bbase + kc * 2 * (COUT * 16), COUT * 16, 128);
          mma_bf16(tmem, ad, bd, IDESC, (tap > 0 || kc > 0) ? 1u : 0u);
        }
      }
      mma_commit(&mbar);
    }
    __syncwarp();
    if (!mbar_wait(&mbar, phase, kSpin)) ok = false;
    phase ^= 1u;
    fence_after_sync();
    __syncthreads();
  }
  if (!ok && lane == 0) atomicExch(a.err, 1);

  // epilogue: warp w owns TMEM lanes / tile pixels [32w, 32w + 32)
  const long long q = q0 + warp * 32 + lane;
  const bool inb = q < a.P;
  const bool inner = inb && interior_pixel(q, a.Hp, a.Wp);
#pragma unroll 1
  for (int c0 = 0; c0 < COUT; c0 += 16) {
    float v[16];
    tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
    if (inb) {
      float m[16];
      if (a.mask && inner) {
        const uint4* mp = reinterpret_cast<const uint4*>(a.mask + q * COUT + c0);
        uint4 mv[2] = {mp[0], mp[1]};
        const bf16* mb = reinterpret_cast<const bf16*>(mv);
#pragma unroll
        for (int i = 0; i < 16; ++i) m[i] = __bfloat162float(mb[i]) > 0.f ? 1.f : 0.f;
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) m[i] = 1.f;
      }
      uint4 ov[2];
      __nv_bfloat162* o2 = reinterpret_cast<__nv_bfloat162*>(ov);
#pragma unroll
      for (int i = 0; i < 16; i += 2) {
        float x0 = v[i], x1 = v[i + 1];
        if (a.bias) { x0 += a.bias[c0 + i]; x1 += a.bias[c0 + i + 1]; }
        if (a.relu) { x0 = fmaxf(x0, 0.f); x1 = fmaxf(x1, 0.f); }
        x0 *= m[i];
        x1 *= m[i + 1];
        if (!inner) { x0 = 0.f; x1 = 0.f; }
        o2[i / 2] = __floats2bfloat162_rn(x0, x1);
      }
      uint4* op = reinterpret_cast<uint4*>(a.out + q * COUT + c0);
      op[0] = ov[0];
      op[1] = ov[1];
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

// ---- elementwise / resampling kernels ------------------------------------------------------
struct LevelGeom {
  int B, H, W, Hp, Wp;  // image size of this level (unpadded H, W)
  __host__ __device__ long long P() const { return (long long)B * Hp * Wp; }
  __device__ long long q(int b, int y, int x) const { return ((long long)b * Hp + y + 1) * Wp + x + 1; }
};

__device__ __forceinline__ void unpack8(const uint4& u, float (&f)[8]) {
  const bf16* p = reinterpret_cast<const bf16*>(&u);
#pragma unroll
  for (int i = 0; i < 8; ++i) f[i] = __bfloat162float(p[i]);
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 u;
  __nv_bfloat162* p = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return u;
}

// decompose a padded pixel index; returns false on the border
__device__ __forceinline__ bool pix(const LevelGeom& g, long long q, int& b, int& y, int& x) {
  const long long img = (long long)g.Hp * g.Wp;
  b = (int)(q / img);
  const int local = (int)(q - (long long)b * img);
  const int yy = local / g.Wp, xx = local - yy * g.Wp;
  y = yy - 1;
  x = xx - 1;
  return yy >= 1 && yy <= g.H && xx >= 1 && xx <= g.W;
}

// out(level l+1) = 2x2 average of in(level l); C channels; one thread per 8 channels
template <int C>
__global__ void pool_kernel(LevelGeom gi, LevelGeom go, const bf16* in, bf16* out) {
  tpf::tc::pdl_trigger();
  constexpr int K = C / 8;
  const long long n = go.P() * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / K;
    const int c = (int)(i - q * K);
    int b, y, x;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (pix(go, q, b, y, x)) {
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) {
          float f[8];
          unpack8(reinterpret_cast<const uint4*>(in + gi.q(b, 2 * y + dy, 2 * x + dx) * C)[c], f);
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[k] += 0.25f * f[k];
        }
    }
    reinterpret_cast<uint4*>(out + q * C)[c] = pack8(acc);
  }
}

// out(level l) = relu(up(t)(level l+1 -> l) + skip)
template <int C>
__global__ void upadd_relu_kernel(LevelGeom gf, LevelGeom gc, const bf16* t, const bf16* skip, bf16* out) {
  tpf::tc::pdl_trigger();
  constexpr int K = C / 8;
  const long long n = gf.P() * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / K;
    const int c = (int)(i - q * K);
    int b, y, x;
    float o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (pix(gf, q, b, y, x)) {
      float f[8], s[8];
      unpack8(reinterpret_cast<const uint4*>(t + gc.q(b, y >> 1, x >> 1) * C)[c], f);
      unpack8(reinterpret_cast<const uint4*>(skip + q * C)[c], s);
#pragma unroll
      for (int k = 0; k < 8; ++k) o[k] = fmaxf(f[k] + s[k], 0.f);
    }
    reinterpret_cast<uint4*>(out + q * C)[c] = pack8(o);
  }
}

// backward of up(): out(level l+1) = 2x2 sum of in(level l)
template <int C>
__global__ void downsum_kernel(LevelGeom gf, LevelGeom gc, const bf16* in, bf16* out) {
  constexpr int K = C / 8;
  const long long n = gc.P() * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / K;
    const int c = (int)(i - q * K);
    int b, y, x;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (pix(gc, q, b, y, x)) {
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) {
          float f[8];
          unpack8(reinterpret_cast<const uint4*>(in + gf.q(b, 2 * y + dy, 2 * x + dx) * C)[c], f);
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[k] += f[k];
        }
    }
    reinterpret_cast<uint4*>(out + q * C)[c] = pack8(acc);
  }
}

// backward of pool() plus the skip gradient, times the ReLU mask of act:
// out(level l) = (0.25 dP(level l+1) + dskip) * (act > 0)
template <int C>
__global__ void pool_bwd_kernel(LevelGeom gf, LevelGeom gc, const bf16* dP, const bf16* dskip, const bf16* act,
                                bf16* out) {
  constexpr int K = C / 8;
  const long long n = gf.P() * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long q = i / K;
    const int c = (int)(i - q * K);
    int b, y, x;
    float o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (pix(gf, q, b, y, x)) {
      float f[8], s[8], m[8];
      unpack8(reinterpret_cast<const uint4*>(dP + gc.q(b, y >> 1, x >> 1) * C)[c], f);
      unpack8(reinterpret_cast<const uint4*>(dskip + q * C)[c], s);
      unpack8(reinterpret_cast<const uint4*>(act + q * C)[c], m);
#pragma unroll
      for (int k = 0; k < 8; ++k) o[k] = (m[k] > 0.f) ? (0.25f * f[k] + s[k]) : 0.f;
    }
    reinterpret_cast<uint4*>(out + q * C)[c] = pack8(o);
  }
}

// input [B][H][W][kIn] FP32 -> xin (16 channels, 0..kIn-1 used)
__global__ void pack_input_kernel(LevelGeom g, const float* in, bf16* xin) {
  tpf::tc::pdl_trigger();
  const long long n = g.P();
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int b, y, x;
    float f0[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float f1[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (pix(g, q, b, y, x)) {
      const long long s = (((long long)b * g.H + y) * g.W + x) * kIn;
#pragma unroll
      for (int c = 0; c < kIn; ++c) f0[c] = in[s + c];
    }
    uint4* o = reinterpret_cast<uint4*>(xin + q * kInPad);
    o[0] = pack8(f0);
    o[1] = pack8(f1);
  }
}

// y[B][H][W] = d0 . w_out + b_out
__global__ void out1x1_kernel(LevelGeom g, const bf16* d0, const float* w, const float* bo, float* yout) {
  const long long n = (long long)g.B * g.H * g.W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.W);
    const long long t = i / g.W;
    const int y = (int)(t % g.H);
    const int b = (int)(t / g.H);
    const uint4* p = reinterpret_cast<const uint4*>(d0 + g.q(b, y, x) * kOutC);
    float f[8], acc = *bo;
    unpack8(p[0], f);
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += f[k] * w[k];
    unpack8(p[1], f);
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += f[k] * w[8 + k];
    yout[i] = acc;
  }
}

// backward of the 1x1 output layer: g_d0 = dy * w * (d0 > 0); gw += sum dy*d0; gb += sum dy
__global__ void out1x1_bwd_kernel(LevelGeom g, const bf16* d0, const float* dy, const float* w, bf16* gd0,
                                  float* gw, float* gb) {
  __shared__ float red[17][8];
  float aw[16], ab = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) aw[k] = 0.f;
  const long long n = g.P();
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    int b, y, x;
    float o0[8] = {0, 0, 0, 0, 0, 0, 0, 0}, o1[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (pix(g, q, b, y, x)) {
      const float d = dy[((long long)b * g.H + y) * g.W + x];
      const uint4* p = reinterpret_cast<const uint4*>(d0 + q * kOutC);
      float f[8];
      unpack8(p[0], f);
#pragma unroll
      for (int k = 0; k < 8; ++k) { aw[k] += d * f[k]; o0[k] = f[k] > 0.f ? d * w[k] : 0.f; }
      unpack8(p[1], f);
#pragma unroll
      for (int k = 0; k < 8; ++k) { aw[8 + k] += d * f[k]; o1[k] = f[k] > 0.f ? d * w[8 + k] : 0.f; }
      ab += d;
    }
    uint4* o = reinterpret_cast<uint4*>(gd0 + q * kOutC);
    o[0] = pack8(o0);
    o[1] = pack8(o1);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 16; ++k) aw[k] = tpf::warp_sum(aw[k]);
  ab = tpf::warp_sum(ab);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 16; ++k) red[k][wid] = aw[k];
    red[16][wid] = ab;
  }
  __syncthreads();
  if (threadIdx.x < 17) {
    float s = 0.f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[threadIdx.x][i];
    if (threadIdx.x < 16) atomicAdd(gw + threadIdx.x, s);
    else atomicAdd(gb, s);
  }
}

// weight (and bias) gradient of a 3x3 convolution on the CUDA cores:
// gW[co][ci][ky][kx] += sum_q dZ[q][co] X[q + (ky-1) Wp + (kx-1)][ci]; gB[co] += sum_q dZ[q][co].
// grid: x = pixel chunks, y = tap, z = (co tile, ci tile); 256 threads = 16 x 16,
// each thread a (TCO/16) x (TCI/16) micro tile.
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) dw_kernel(const bf16* X, const bf16* dZ, float* gW, float* gB, long long P,
                                                 int Wp, int cin_logical, int chunk) {
  constexpr int TCO = COUT < 64 ? COUT : 64;
  constexpr int TCI = CIN < 64 ? CIN : 64;
  constexpr int MCO = TCO / 16, MCI = TCI / 16;
  constexpr int SUB = 32;
  __shared__ float sZ[SUB][TCO + 1];
  __shared__ float sX[SUB][TCI + 1];
  const int tap = blockIdx.y;
  const int nci_t = CIN / TCI;
  const int co0 = (blockIdx.z / nci_t) * TCO, ci0 = (blockIdx.z % nci_t) * TCI;
  const long long shift = (long long)(tap / 3 - 1) * Wp + (tap % 3 - 1);
  const int tco = threadIdx.x >> 4, tci = threadIdx.x & 15;
  float acc[MCO][MCI];
  float bacc[MCO];
#pragma unroll
  for (int i = 0; i < MCO; ++i) {
    bacc[i] = 0.f;
#pragma unroll
    for (int j = 0; j < MCI; ++j) acc[i][j] = 0.f;
  }
  const long long p_begin = (long long)blockIdx.x * chunk;
  const long long p_end = min(P, p_begin + chunk);
  for (long long p0 = p_begin; p0 < p_end; p0 += SUB) {
    for (int i = threadIdx.x; i < SUB * TCO; i += 256) {
      const int r = i / TCO, c = i - r * TCO;
      const long long q = p0 + r;
      sZ[r][c] = (q < p_end) ? __bfloat162float(dZ[q * COUT + co0 + c]) : 0.f;
    }
    for (int i = threadIdx.x; i < SUB * TCI; i += 256) {
      const int r = i / TCI, c = i - r * TCI;
      const long long q = p0 + r, qs = q + shift;
      sX[r][c] = (q < p_end && qs >= 0 && qs < P) ? __bfloat162float(X[qs * CIN + ci0 + c]) : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < SUB; ++r) {
      float z[MCO], xv[MCI];
#pragma unroll
      for (int i = 0; i < MCO; ++i) z[i] = sZ[r][tco + 16 * i];
#pragma unroll
      for (int j = 0; j < MCI; ++j) xv[j] = sX[r][tci + 16 * j];
#pragma unroll
      for (int i = 0; i < MCO; ++i) {
        bacc[i] += z[i];
#pragma unroll
        for (int j = 0; j < MCI; ++j) acc[i][j] += z[i] * xv[j];
      }
    }
    __syncthreads();
  }
  const int ky = tap / 3, kx = tap % 3;
#pragma unroll
  for (int i = 0; i < MCO; ++i) {
    const int co = co0 + tco + 16 * i;
#pragma unroll
    for (int j = 0; j < MCI; ++j) {
      const int ci = ci0 + tci + 16 * j;
      if (ci < cin_logical) atomicAdd(gW + (((size_t)co * cin_logical + ci) * 3 + ky) * 3 + kx, acc[i][j]);
    }
    if (tap == 4 && ci0 == 0 && tci == 0) atomicAdd(gB + co, bacc[i]);
  }
}

// forward weights [9][CIN/8][COUT][8] and transposed/flipped backward-data
// weights [9][COUT/8][CIN][8] (bwd: a convolution from COUT to CIN channels)
__global__ void arrange_kernel(const float* W, int cin_logical, int cin, int cout, bf16* wf, bf16* wb) {
  const int n = 9 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    // forward element i = ((tap * (cin/8) + cb) * cout + co) * 8 + j
    {
      const int j = i & 7;
      int r = i >> 3;
      const int co = r % cout;
      r /= cout;
      const int cb = r % (cin / 8);
      const int tap = r / (cin / 8);
      const int ci = cb * 8 + j;
      const float v = (ci < cin_logical) ? W[((size_t)co * cin_logical + ci) * 9 + tap] : 0.f;
      wf[i] = __float2bfloat16_rn(v);
    }
    if (wb) {
      // backward element i = ((tap' * (cout/8) + cb') * cin + ci) * 8 + j, co = cb'*8 + j, tap = 8 - tap'
      const int j = i & 7;
      int r = i >> 3;
      const int ci = r % cin;
      r /= cin;
      const int cb = r % (cout / 8);
      const int tapb = r / (cout / 8);
      const int co = cb * 8 + j;
      const float v = (ci < cin_logical) ? W[((size_t)co * cin_logical + ci) * 9 + (8 - tapb)] : 0.f;
      wb[i] = __float2bfloat16_rn(v);
    }
  }
}

// per-sample relative squared error L_b = sum (y - t)^2 / sum t^2 -> sums[2b], sums[2b+1]
__global__ void loss_sums_kernel(int B, long long npix, const float* y, const float* t, double* sums) {
  const int b = blockIdx.y;
  double e = 0.0, s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x) {
    const double d = (double)y[b * npix + i] - t[b * npix + i];
    e += d * d;
    s += (double)t[b * npix + i] * t[b * npix + i];
  }
  double v[2] = {e, s};
  __shared__ double scratch[2 * 32];
  tpf::block_sum<2>(v, scratch);
  if (threadIdx.x == 0) {
    atomicAdd(sums + 2 * b, v[0]);
    atomicAdd(sums + 2 * b + 1, v[1]);
  }
}

// dy = 2 (y - t) / (B * sum t^2)
__global__ void loss_grad_kernel(int B, long long npix, const float* y, const float* t, const double* sums,
                                 float* dy) {
  const long long n = (long long)B * npix;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / npix);
    const double s = sums[2 * b + 1] > 0.0 ? sums[2 * b + 1] : 1.0;
    dy[i] = (float)(2.0 * ((double)y[i] - t[i]) / (B * s));
  }
}

// Energy loss of a coarse-grid correction (two-level preconditioner training):
// per sample b, with y the network output on the coarse image, x = in[..,0]
// the scaled coarse residual and A~ = I - (couplings c0 to the next row, c1 to
// the next column; unit diagonal inside the nc0 x nc1 coarse grid),
//   L_b = (y.A~y - 2 y.x) / E_b + 1  = ||e1 - P y^||_A^2 / ||e1||_A^2,
// dL/dy = 2 (A~y - x) / (B E_b).  Pixels outside the coarse grid carry no term.
__global__ void energy_terms_kernel(int B, int H, int W, int nc0, int nc1, const float* y, const float* in2,
                                    const float* coupl, double* sums, float* dy, const double* escale,
                                    int want_grad) {
  const int b = blockIdx.y;
  const long long npix = (long long)H * W;
  const float* yb = y + b * npix;
  const float* xb = in2 + b * npix * kIn;
  const float* cb = coupl + b * npix * 2;
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npix; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / W), j = (int)(q - (long long)i * W);
    float g = 0.f;
    if (i < nc0 && j < nc1) {
      const float yv = yb[q];
      float ay = yv;
      if (i + 1 < nc0) ay -= cb[2 * q] * yb[q + W];
      if (i > 0) ay -= cb[2 * (q - W)] * yb[q - W];
      if (j + 1 < nc1) ay -= cb[2 * q + 1] * yb[q + 1];
      if (j > 0) ay -= cb[2 * (q - 1) + 1] * yb[q - 1];
      const float xv = xb[kIn * q];
      acc += (double)yv * ((double)ay - 2.0 * (double)xv);
      g = ay - xv;
    }
    if (want_grad) dy[b * npix + q] = (float)(2.0 * g / (B * escale[b]));
  }
  double v[1] = {acc};
  __shared__ double scratch[32];
  tpf::block_sum<1>(v, scratch);
  if (threadIdx.x == 0) atomicAdd(sums + b, v[0]);
}

__global__ void adam_kernel(float* p, float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2, float wd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.f;
  }
}

inline int grid_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}

// ---- conv dispatch ---------------------------------------------------------------------------
template <int CIN, int COUT>
int launch_conv_t(const ConvArgs& a, cudaStream_t s) {
  constexpr int smem = conv_smem_bytes(CIN, COUT);
  static bool attr = false;
  if (!attr) {
    TPF_CUDA_TRY(cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    attr = true;
  }
  const long long tiles = (a.P + kTile - 1) / kTile;
  // programmatic dependent launch: the prologue overlaps the previous kernel,
  // whose outputs are read only after griddepcontrol.wait
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)tiles);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl;
  cfg.numAttrs = 1;
  TPF_CUDA_TRY(cudaLaunchKernelEx(&cfg, conv3x3_tc_kernel<CIN, COUT>, a));
  return TPF_OK;
}

#define TPF_CONV_CASES(X) \
  X(16, 16) X(16, 32) X(32, 16) X(32, 32) X(32, 64) X(64, 32) X(64, 64) X(64, 128) X(128, 64) X(128, 128)

int launch_conv(int cin, int cout, const ConvArgs& a, cudaStream_t s) {
#define TPF_CONV_CASE(ci, co) \
  if (cin == ci && cout == co) return launch_conv_t<ci, co>(a, s);
  TPF_CONV_CASES(TPF_CONV_CASE)
#undef TPF_CONV_CASE
  tpf::set_error("no convolution kernel for %d -> %d channels", cin, cout);
  return TPF_EINVAL;
}

int launch_dw(int cin, int cout, const bf16* X, const bf16* dZ, float* gW, float* gB, long long P, int Wp,
              int cin_logical, cudaStream_t s) {
  const int chunk = 2048;
  const unsigned nx = (unsigned)((P + chunk - 1) / chunk);
#define TPF_DW_CASE(ci, co)                                                                    \
  if (cin == ci && cout == co) {                                                               \
    constexpr int TCO = co < 64 ? co : 64, TCI = ci < 64 ? ci : 64;                           \
    dim3 grid(nx, 9, (co / TCO) * (ci / TCI));                                                 \
    dw_kernel<ci, co><<<grid, 256, 0, s>>>(X, dZ, gW, gB, P, Wp, cin_logical, chunk);          \
    TPF_CUDA_TRY(cudaGetLastError());                                                          \
    return TPF_OK;                                                                             \
  }
  TPF_CONV_CASES(TPF_DW_CASE)
#undef TPF_DW_CASE
  tpf::set_error("no weight-gradient kernel for %d -> %d channels", cin, cout);
  return TPF_EINVAL;
}

#define TPF_CH_DISPATCH(C, CALL) \
  switch (C) {                   \
    case 16: CALL(16); break;    \
    case 32: CALL(32); break;    \
    case 64: CALL(64); break;    \
    case 128: CALL(128); break;  \
    default: break;              \
  }

}  // namespace

// ============================================================================================
struct tpf_unet {
  int H = 0, W = 0, max_batch = 0;
  float* params = nullptr;
  float* grads = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  long long adam_t = 0;
  bf16* wf[kConvs] = {};
  bf16* wb[kConvs] = {};
  bool arranged = false;
  // forward activations
  bf16 *xin = nullptr, *e0a = nullptr, *e0 = nullptr, *p0 = nullptr, *e1a = nullptr, *e1 = nullptr, *p1 = nullptr,
       *e2a = nullptr, *e2 = nullptr, *p2 = nullptr, *e3a = nullptr, *e3 = nullptr, *t2 = nullptr, *d2a = nullptr,
       *d2 = nullptr, *t1 = nullptr, *d1a = nullptr, *d1 = nullptr, *t0 = nullptr, *d0a = nullptr, *d0 = nullptr;
  float* out = nullptr;
  // backward
  bf16 *g_d0 = nullptr, *g_d0a = nullptr, *g_e0 = nullptr, *g_e0a = nullptr, *g_t0 = nullptr, *g_d1 = nullptr,
       *g_d1a = nullptr, *g_p0 = nullptr, *g_e1 = nullptr, *g_e1a = nullptr, *g_t1 = nullptr, *g_d2 = nullptr,
       *g_d2a = nullptr, *g_p1 = nullptr, *g_e2 = nullptr, *g_e2a = nullptr, *g_t2 = nullptr, *g_e3 = nullptr,
       *g_e3a = nullptr, *g_p2 = nullptr;
  float* dy = nullptr;
  double* sums = nullptr;
  int* err = nullptr;
  bool training_buffers = false;
  int last_batch = 0;
  std::vector<void*> allocs;

  LevelGeom geom(int l, int B) const {
    LevelGeom g;
    g.B = B;
    g.H = H >> l;
    g.W = W >> l;
    g.Hp = g.H + 2;
    g.Wp = g.W + 2;
    return g;
  }
};

namespace {

template <typename T>
int ualloc(tpf_unet* n, T** p, size_t count) {
  if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    tpf::set_error("cudaMalloc of %zu bytes failed", count * sizeof(T));
    return TPF_ECUDA;
  }
  n->allocs.push_back(*p);
  return TPF_OK;
}

int act_alloc(tpf_unet* n, bf16** p, int level, int C) {
  const LevelGeom g = n->geom(level, n->max_batch);
  int st = ualloc(n, p, (size_t)g.P() * C);
  if (st) return st;
  TPF_CUDA_TRY(cudaMemset(*p, 0, (size_t)g.P() * C * sizeof(bf16)));
  return TPF_OK;
}

int ensure_training(tpf_unet* n) {
  if (n->training_buffers) return TPF_OK;
  int st = 0;
  struct A { bf16** p; int l, c; };
  A list[] = {{&n->g_d0, 0, 16}, {&n->g_d0a, 0, 16}, {&n->g_e0, 0, 16}, {&n->g_e0a, 0, 16},
              {&n->g_t0, 1, 16}, {&n->g_d1, 1, 32},  {&n->g_d1a, 1, 32}, {&n->g_p0, 1, 16},
              {&n->g_e1, 1, 32}, {&n->g_e1a, 1, 32}, {&n->g_t1, 2, 32},  {&n->g_d2, 2, 64},
              {&n->g_d2a, 2, 64}, {&n->g_p1, 2, 32}, {&n->g_e2, 2, 64},  {&n->g_e2a, 2, 64},
              {&n->g_t2, 3, 64}, {&n->g_e3, 3, 128}, {&n->g_e3a, 3, 128}, {&n->g_p2, 3, 64}};
  for (auto& a : list)
    if ((st = act_alloc(n, a.p, a.l, a.c))) return st;
  const int64_t np = layout().total;
  if ((st = ualloc(n, &n->grads, np)) || (st = ualloc(n, &n->m, np)) || (st = ualloc(n, &n->v, np))) return st;
  TPF_CUDA_TRY(cudaMemset(n->grads, 0, np * sizeof(float)));
  TPF_CUDA_TRY(cudaMemset(n->m, 0, np * sizeof(float)));
  TPF_CUDA_TRY(cudaMemset(n->v, 0, np * sizeof(float)));
  if ((st = ualloc(n, &n->dy, (size_t)n->max_batch * n->H * n->W))) return st;
  if ((st = ualloc(n, &n->sums, 2 * (size_t)n->max_batch))) return st;
  n->training_buffers = true;
  return TPF_OK;
}

int arrange(tpf_unet* n, cudaStream_t s) {
  const ParamLayout& L = layout();
  for (int l = 0; l < kConvs; ++l) {
    const int ck = cin_kernel(l), co = kLayers[l].cout;
    arrange_kernel<<<grid_for(9 * ck * co), 256, 0, s>>>(n->params + L.w[l], kLayers[l].cin, ck, co, n->wf[l],
                                                          l == 0 ? nullptr : n->wb[l]);
  }
  TPF_CUDA_TRY(cudaGetLastError());
  n->arranged = true;
  return TPF_OK;
}

int conv(tpf_unet* n, int l, int B, const bf16* in, bf16* out, cudaStream_t s) {
  const ParamLayout& L = layout();
  const LevelGeom g = n->geom(kLayers[l].level, B);
  ConvArgs a{};
  a.in = in;
  a.out = out;
  a.w = n->wf[l];
  a.bias = n->params + L.b[l];
  a.mask = nullptr;
  a.P = g.P();
  a.Hp = g.Hp;
  a.Wp = g.Wp;
  a.relu = kLayers[l].relu;
  a.err = n->err;
  return launch_conv(cin_kernel(l), kLayers[l].cout, a, s);
}

// backward data of layer l: out = conv^T(dz) * (mask > 0) (mask may be null)
int conv_bwd(tpf_unet* n, int l, int B, const bf16* dz, const bf16* mask, bf16* out, cudaStream_t s) {
  const LevelGeom g = n->geom(kLayers[l].level, B);
  ConvArgs a{};
  a.in = dz;
  a.out = out;
  a.w = n->wb[l];
  a.bias = nullptr;
  a.mask = mask;
  a.P = g.P();
  a.Hp = g.Hp;
  a.Wp = g.Wp;
  a.relu = 0;
  a.err = n->err;
  return launch_conv(kLayers[l].cout, cin_kernel(l), a, s);
}

int wgrad(tpf_unet* n, int l, int B, const bf16* X, const bf16* dz, cudaStream_t s) {
  const ParamLayout& L = layout();
  const LevelGeom g = n->geom(kLayers[l].level, B);
  return launch_dw(cin_kernel(l), kLayers[l].cout, X, dz, n->grads + L.w[l], n->grads + L.b[l], g.P(), g.Wp,
                   kLayers[l].cin, s);
}

template <int C>
void pool_t(const LevelGeom& gi, const LevelGeom& go, const bf16* in, bf16* out, cudaStream_t s) {
  pool_kernel<C><<<grid_for(go.P() * (C / 8)), 256, 0, s>>>(gi, go, in, out);
}
template <int C>
void upadd_t(const LevelGeom& gf, const LevelGeom& gc, const bf16* t, const bf16* sk, bf16* out, cudaStream_t s) {
  upadd_relu_kernel<C><<<grid_for(gf.P() * (C / 8)), 256, 0, s>>>(gf, gc, t, sk, out);
}
template <int C>
void downsum_t(const LevelGeom& gf, const LevelGeom& gc, const bf16* in, bf16* out, cudaStream_t s) {
  downsum_kernel<C><<<grid_for(gc.P() * (C / 8)), 256, 0, s>>>(gf, gc, in, out);
}
template <int C>
void poolbwd_t(const LevelGeom& gf, const LevelGeom& gc, const bf16* dP, const bf16* sk, const bf16* act, bf16* out,
               cudaStream_t s) {
  pool_bwd_kernel<C><<<grid_for(gf.P() * (C / 8)), 256, 0, s>>>(gf, gc, dP, sk, act, out);
}

int forward(tpf_unet* n, int B, cudaStream_t s) {
  int st;
  if (!n->arranged && (st = arrange(n, s))) return st;
  const LevelGeom g0 = n->geom(0, B), g1 = n->geom(1, B), g2 = n->geom(2, B), g3 = n->geom(3, B);
  if ((st = conv(n, 0, B, n->xin, n->e0a, s)) || (st = conv(n, 1, B, n->e0a, n->e0, s))) return st;
  pool_t<16>(g0, g1, n->e0, n->p0, s);
  if ((st = conv(n, 2, B, n->p0, n->e1a, s)) || (st = conv(n, 3, B, n->e1a, n->e1, s))) return st;
  pool_t<32>(g1, g2, n->e1, n->p1, s);
  if ((st = conv(n, 4, B, n->p1, n->e2a, s)) || (st = conv(n, 5, B, n->e2a, n->e2, s))) return st;
  pool_t<64>(g2, g3, n->e2, n->p2, s);
  if ((st = conv(n, 6, B, n->p2, n->e3a, s)) || (st = conv(n, 7, B, n->e3a, n->e3, s))) return st;
  if ((st = conv(n, 8, B, n->e3, n->t2, s))) return st;
  upadd_t<64>(g2, g3, n->t2, n->e2, n->d2a, s);
  if ((st = conv(n, 9, B, n->d2a, n->d2, s)) || (st = conv(n, 10, B, n->d2, n->t1, s))) return st;
  upadd_t<32>(g1, g2, n->t1, n->e1, n->d1a, s);
  if ((st = conv(n, 11, B, n->d1a, n->d1, s)) || (st = conv(n, 12, B, n->d1, n->t0, s))) return st;
  upadd_t<16>(g0, g1, n->t0, n->e0, n->d0a, s);
  if ((st = conv(n, 13, B, n->d0a, n->d0, s))) return st;
  const ParamLayout& L = layout();
  out1x1_kernel<<<grid_for((long long)B * n->H * n->W), 256, 0, s>>>(g0, n->d0, n->params + L.wo, n->params + L.bo,
                                                                     n->out);
  TPF_CUDA_TRY(cudaGetLastError());
  n->last_batch = B;
  return TPF_OK;
}

// gradients of all parameters (accumulated into n->grads) for dy = dL/dy of the last forward
int backward(tpf_unet* n, int B, const float* dy, cudaStream_t s) {
  int st;
  if ((st = ensure_training(n))) return st;
  const ParamLayout& L = layout();
  const LevelGeom g0 = n->geom(0, B), g1 = n->geom(1, B), g2 = n->geom(2, B), g3 = n->geom(3, B);
  out1x1_bwd_kernel<<<grid_for(g0.P()), 256, 0, s>>>(g0, n->d0, dy, n->params + L.wo, n->g_d0, n->grads + L.wo,
                                                     n->grads + L.bo);
  TPF_CUDA_TRY(cudaGetLastError());
  // level 0 decoder
  if ((st = wgrad(n, 13, B, n->d0a, n->g_d0, s)) || (st = conv_bwd(n, 13, B, n->g_d0, n->d0a, n->g_d0a, s)))
    return st;
  downsum_t<16>(g0, g1, n->g_d0a, n->g_t0, s);
  if ((st = wgrad(n, 12, B, n->d1, n->g_t0, s)) || (st = conv_bwd(n, 12, B, n->g_t0, n->d1, n->g_d1, s))) return st;
  if ((st = wgrad(n, 11, B, n->d1a, n->g_d1, s)) || (st = conv_bwd(n, 11, B, n->g_d1, n->d1a, n->g_d1a, s)))
    return st;
  downsum_t<32>(g1, g2, n->g_d1a, n->g_t1, s);
  if ((st = wgrad(n, 10, B, n->d2, n->g_t1, s)) || (st = conv_bwd(n, 10, B, n->g_t1, n->d2, n->g_d2, s))) return st;
  if ((st = wgrad(n, 9, B, n->d2a, n->g_d2, s)) || (st = conv_bwd(n, 9, B, n->g_d2, n->d2a, n->g_d2a, s))) return st;
  downsum_t<64>(g2, g3, n->g_d2a, n->g_t2, s);
  if ((st = wgrad(n, 8, B, n->e3, n->g_t2, s)) || (st = conv_bwd(n, 8, B, n->g_t2, n->e3, n->g_e3, s))) return st;
  if ((st = wgrad(n, 7, B, n->e3a, n->g_e3, s)) || (st = conv_bwd(n, 7, B, n->g_e3, n->e3a, n->g_e3a, s))) return st;
  if ((st = wgrad(n, 6, B, n->p2, n->g_e3a, s)) || (st = conv_bwd(n, 6, B, n->g_e3a, nullptr, n->g_p2, s)))
    return st;
  poolbwd_t<64>(g2, g3, n->g_p2, n->g_d2a, n->e2, n->g_e2, s);
  if ((st = wgrad(n, 5, B, n->e2a, n->g_e2, s)) || (st = conv_bwd(n, 5, B, n->g_e2, n->e2a, n->g_e2a, s))) return st;
  if ((st = wgrad(n, 4, B, n->p1, n->g_e2a, s)) || (st = conv_bwd(n, 4, B, n->g_e2a, nullptr, n->g_p1, s)))
    return st;
  poolbwd_t<32>(g1, g2, n->g_p1, n->g_d1a, n->e1, n->g_e1, s);
  if ((st = wgrad(n, 3, B, n->e1a, n->g_e1, s)) || (st = conv_bwd(n, 3, B, n->g_e1, n->e1a, n->g_e1a, s))) return st;
  if ((st = wgrad(n, 2, B, n->p0, n->g_e1a, s)) || (st = conv_bwd(n, 2, B, n->g_e1a, nullptr, n->g_p0, s)))
    return st;
  poolbwd_t<16>(g0, g1, n->g_p0, n->g_d0a, n->e0, n->g_e0, s);
  if ((st = wgrad(n, 1, B, n->e0a, n->g_e0, s)) || (st = conv_bwd(n, 1, B, n->g_e0, n->e0a, n->g_e0a, s))) return st;
  if ((st = wgrad(n, 0, B, n->xin, n->g_e0a, s))) return st;
  TPF_CUDA_TRY(cudaGetLastError());
  return TPF_OK;
}

int check_err(tpf_unet* n, cudaStream_t s) {
  int herr = 0;
  TPF_CUDA_TRY(cudaMemcpyAsync(&herr, n->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPF_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) {
    tpf::set_error("a tensor-core convolution wait timed out");
    return TPF_EABORT;
  }
  return TPF_OK;
}

}  // namespace

// ---- internal interface for the learned PPE solver ---------------------------------------------
namespace tpf {
int unet_dims(const tpf_unet* n, int* H, int* W, int* max_batch) {
  *H = n->H;
  *W = n->W;
  *max_batch = n->max_batch;
  return TPF_OK;
}
bf16* unet_input(tpf_unet* n) { return n->xin; }
const float* unet_output(tpf_unet* n) { return n->out; }
int unet_forward_packed(tpf_unet* n, int B, cudaStream_t s) { return forward(n, B, s); }
int unet_prepare_weights(tpf_unet* n, cudaStream_t s) { return n->arranged ? TPF_OK : arrange(n, s); }
int unet_check(tpf_unet* n, cudaStream_t s) { return check_err(n, s); }
}  // namespace tpf

// ============================================================================================
extern "C" {

int64_t tpf_unet_num_params(void) { return layout().total; }

int tpf_unet_create(tpf_unet** out, int H, int W, int max_batch) {
  TPF_CHECK_ARG(out != nullptr, "null handle pointer");
  TPF_CHECK_ARG(H >= 8 && W >= 8 && H % 8 == 0 && W % 8 == 0, "U-Net image size must be a multiple of 8 (got %dx%d)",
                H, W);
  TPF_CHECK_ARG(max_batch >= 1, "max_batch must be >= 1");
  auto* n = new tpf_unet();
  n->H = H;
  n->W = W;
  n->max_batch = max_batch;
  int st = 0;
  const ParamLayout& L = layout();
  auto fail = [&](int code) {
    for (void* p : n->allocs) cudaFree(p);
    delete n;
    return code;
  };
  if ((st = ualloc(n, &n->params, L.total))) return fail(st);
  TPF_CUDA_TRY(cudaMemset(n->params, 0, L.total * sizeof(float)));
  for (int l = 0; l < kConvs; ++l) {
    const size_t cnt = (size_t)9 * cin_kernel(l) * kLayers[l].cout;
    if ((st = ualloc(n, &n->wf[l], cnt))) return fail(st);
    if (l > 0 && (st = ualloc(n, &n->wb[l], cnt))) return fail(st);
  }
  struct A { bf16** p; int l, c; };
  A list[] = {{&n->xin, 0, 16}, {&n->e0a, 0, 16}, {&n->e0, 0, 16},   {&n->p0, 1, 16},  {&n->e1a, 1, 32},
              {&n->e1, 1, 32},  {&n->p1, 2, 32},  {&n->e2a, 2, 64},  {&n->e2, 2, 64},  {&n->p2, 3, 64},
              {&n->e3a, 3, 128}, {&n->e3, 3, 128}, {&n->t2, 3, 64},  {&n->d2a, 2, 64}, {&n->d2, 2, 64},
              {&n->t1, 2, 32},  {&n->d1a, 1, 32}, {&n->d1, 1, 32},   {&n->t0, 1, 16},  {&n->d0a, 0, 16},
              {&n->d0, 0, 16}};
  for (auto& a : list)
    if ((st = act_alloc(n, a.p, a.l, a.c))) return fail(st);
  if ((st = ualloc(n, &n->out, (size_t)max_batch * H * W))) return fail(st);
  if ((st = ualloc(n, &n->err, 1))) return fail(st);
  TPF_CUDA_TRY(cudaMemset(n->err, 0, sizeof(int)));
  *out = n;
  return TPF_OK;
}

int tpf_unet_destroy(tpf_unet* n) {
  if (!n) return TPF_OK;
  cudaDeviceSynchronize();
  for (void* p : n->allocs) cudaFree(p);
  delete n;
  return TPF_OK;
}

int tpf_unet_set_params(tpf_unet* n, const float* params, int on_device) {
  TPF_CHECK_ARG(n && params, "null argument");
  TPF_CUDA_TRY(cudaMemcpy(n->params, params, layout().total * sizeof(float),
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
  n->arranged = false;
  n->adam_t = 0;
  if (n->training_buffers) {
    TPF_CUDA_TRY(cudaMemset(n->m, 0, layout().total * sizeof(float)));
    TPF_CUDA_TRY(cudaMemset(n->v, 0, layout().total * sizeof(float)));
    TPF_CUDA_TRY(cudaMemset(n->grads, 0, layout().total * sizeof(float)));
  }
  return TPF_OK;
}

int tpf_unet_get_params(tpf_unet* n, float* params, int on_device) {
  TPF_CHECK_ARG(n && params, "null argument");
  TPF_CUDA_TRY(cudaMemcpy(params, n->params, layout().total * sizeof(float),
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
  return TPF_OK;
}

int tpf_unet_forward(tpf_unet* n, int B, const float* in2, float* y, void* stream) {
  TPF_CHECK_ARG(n && in2 && y, "null argument");
  TPF_CHECK_ARG(B >= 1 && B <= n->max_batch, "batch %d outside [1, %d]", B, n->max_batch);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const LevelGeom g0 = n->geom(0, B);
  pack_input_kernel<<<grid_for(g0.P()), 256, 0, s>>>(g0, in2, n->xin);
  TPF_CUDA_TRY(cudaGetLastError());
  int st = forward(n, B, s);
  if (st) return st;
  TPF_CUDA_TRY(cudaMemcpyAsync(y, n->out, sizeof(float) * B * n->H * n->W, cudaMemcpyDeviceToDevice, s));
  return check_err(n, s);
}

int tpf_unet_backward(tpf_unet* n, int B, const float* dy, float* grads, void* stream) {
  TPF_CHECK_ARG(n && dy, "null argument");
  TPF_CHECK_ARG(B == n->last_batch, "backward needs the activations of a forward pass with the same batch");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = ensure_training(n);
  if (st) return st;
  TPF_CUDA_TRY(cudaMemsetAsync(n->grads, 0, layout().total * sizeof(float), s));
  if ((st = backward(n, B, dy, s))) return st;
  if (grads)
    TPF_CUDA_TRY(cudaMemcpyAsync(grads, n->grads, layout().total * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return check_err(n, s);
}

int tpf_unet_train_step(tpf_unet* n, int B, const float* in2, const float* target, float lr, float weight_decay,
                        double* loss, void* stream) {
  TPF_CHECK_ARG(n && in2 && target, "null argument");
  TPF_CHECK_ARG(B >= 1 && B <= n->max_batch, "batch %d outside [1, %d]", B, n->max_batch);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = ensure_training(n);
  if (st) return st;
  const LevelGeom g0 = n->geom(0, B);
  pack_input_kernel<<<grid_for(g0.P()), 256, 0, s>>>(g0, in2, n->xin);
  if ((st = forward(n, B, s))) return st;
  const long long npix = (long long)n->H * n->W;
  TPF_CUDA_TRY(cudaMemsetAsync(n->sums, 0, 2 * sizeof(double) * B, s));
  loss_sums_kernel<<<dim3(64, B), 256, 0, s>>>(B, npix, n->out, target, n->sums);
  loss_grad_kernel<<<grid_for(B * npix), 256, 0, s>>>(B, npix, n->out, target, n->sums, n->dy);
  TPF_CUDA_TRY(cudaGetLastError());
  if ((st = backward(n, B, n->dy, s))) return st;
  n->adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)n->adam_t), c2 = 1.f - std::pow(b2, (float)n->adam_t);
  adam_kernel<<<grid_for(layout().total), 256, 0, s>>>(n->params, n->grads, n->m, n->v, layout().total, lr, b1, b2,
                                                        1e-8f, c1, c2, weight_decay);
  TPF_CUDA_TRY(cudaGetLastError());
  n->arranged = false;
  if (loss) {
    std::vector<double> hs(2 * B);
    TPF_CUDA_TRY(cudaMemcpyAsync(hs.data(), n->sums, 2 * sizeof(double) * B, cudaMemcpyDeviceToHost, s));
    if ((st = check_err(n, s))) return st;
    double L = 0.0;
    for (int b = 0; b < B; ++b) L += hs[2 * b] / (hs[2 * b + 1] > 0 ? hs[2 * b + 1] : 1.0);
    *loss = L / B;
    return TPF_OK;
  }
  return TPF_OK;
}

int tpf_unet_train_step_energy(tpf_unet* n, int B, const float* in2, const float* coupl, const double* escale,
                               int nc0, int nc1, float lr, float weight_decay, double* loss, void* stream) {
  TPF_CHECK_ARG(n && in2 && coupl && escale, "null argument");
  TPF_CHECK_ARG(B >= 1 && B <= n->max_batch, "batch %d outside [1, %d]", B, n->max_batch);
  TPF_CHECK_ARG(nc0 >= 1 && nc1 >= 1 && nc0 <= n->H && nc1 <= n->W, "coarse grid %dx%d outside the image", nc0, nc1);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int st = ensure_training(n);
  if (st) return st;
  const LevelGeom g0 = n->geom(0, B);
  pack_input_kernel<<<grid_for(g0.P()), 256, 0, s>>>(g0, in2, n->xin);
  if ((st = forward(n, B, s))) return st;
  TPF_CUDA_TRY(cudaMemsetAsync(n->sums, 0, sizeof(double) * B, s));
  energy_terms_kernel<<<dim3(64, B), 256, 0, s>>>(B, n->H, n->W, nc0, nc1, n->out, in2, coupl, n->sums, n->dy,
                                                  escale, 1);
  TPF_CUDA_TRY(cudaGetLastError());
  if ((st = backward(n, B, n->dy, s))) return st;
  n->adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)n->adam_t), c2 = 1.f - std::pow(b2, (float)n->adam_t);
  adam_kernel<<<grid_for(layout().total), 256, 0, s>>>(n->params, n->grads, n->m, n->v, layout().total, lr, b1, b2,
                                                        1e-8f, c1, c2, weight_decay);
  TPF_CUDA_TRY(cudaGetLastError());
  n->arranged = false;
  if (loss) {
    std::vector<double> hs(B), he(B);
    TPF_CUDA_TRY(cudaMemcpyAsync(hs.data(), n->sums, sizeof(double) * B, cudaMemcpyDeviceToHost, s));
    TPF_CUDA_TRY(cudaMemcpyAsync(he.data(), escale, sizeof(double) * B, cudaMemcpyDeviceToHost, s));
    if ((st = check_err(n, s))) return st;
    double L = 0.0;
    for (int b = 0; b < B; ++b) L += hs[b] / (he[b] > 0 ? he[b] : 1.0) + 1.0;
    *loss = L / B;
  }
  return TPF_OK;
}

}  // extern "C"

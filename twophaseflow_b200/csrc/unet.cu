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

#include <cuda.h>   // CUtensorMap and its enums (the encoder is fetched through the runtime)
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

// Three input windows (rows dy = -1, 0, +1 of 130 pixels, zero outside the
// batch) in channel-plane layout: plane c holds channels [8c, 8c+8) of the
// 130 pixels as 16-byte rows (K-major SWIZZLE_NONE core matrices).  Lanes
// 8k..8k+7 of a warp take 8 consecutive pixels of one channel chunk, so each
// warp writes whole 128-byte plane rows (no shared-memory bank conflicts;
// the plane stride of 2080 bytes would otherwise put 8 lanes on the same
// banks) and reads whole 32-byte sectors of the pixel-major input.  For
// 128-thread CTAs.
template <int CIN>
__device__ __forceinline__ void load_windows(const bf16* in, long long P, int Wp, long long q0, unsigned char* sA) {
  constexpr int KCH = CIN / 8;
  constexpr int WIN_BYTES = KCH * kPlane;
  constexpr int N = ((kWin + 7) / 8) * KCH * 8;   // 17 blocks of 8 pixels x chunks x 8 lanes
#pragma unroll 1
  for (int w = 0; w < 3; ++w) {
    const long long qw = q0 - 1 + (long long)(w - 1) * Wp;
    for (int i = threadIdx.x; i < N; i += 128) {
      const int rest = i >> 3;
      const int c = rest % KCH, j = (rest / KCH) * 8 + (i & 7);
      if (j < kWin) {
        const long long q = qw + j;
        const bool valid = (q >= 0 && q < P);
        tpf::tc::cp_async16(sA + w * WIN_BYTES + c * kPlane + j * 16, in + (valid ? q : 0) * CIN + c * 8, valid);
      }
    }
  }
  tpf::tc::cp_async_commit();
}

// ---- tensor-copy-fed convolution (the layered forward and backward-data path) ---------------
// The three input windows come straight from the pixel-major activations by
// tiled tensor copies: a window block is [130 pixels][R bytes], R = 2 min(CIN,
// 64) = 32, 64 or 128 (channels [64 kb, 64 kb + R/2) of each pixel), written
// with the R-byte swizzle, which is the K-major swizzled operand layout of the
// MMA with one pixel per row; tap dx is the same block read from row dx on.
// Pixels outside the batch are zero-filled by the copy.  Weights are one
// bulk copy per (tap, 8-channel plane) of the CTA's NS output channels
// ([9][CIN/8][NS][8], K-major SWIZZLE_NONE core matrices), or a single copy
// when NS = COUT.  The grid's y dimension splits COUT into NS-wide slices so
// that the small deep-level images still occupy dozens of SMs.
template <int CIN>
struct WinGeom {
  static constexpr int R = CIN < 64 ? CIN * 2 : 128;               // bytes of a block row
  static constexpr int KB = CIN < 64 ? 1 : CIN / 64;               // blocks per window
  static constexpr int BLOCK = ((kWin * R + 1023) / 1024) * 1024;  // 1024-byte aligned block
  static constexpr int BYTES = 3 * KB * BLOCK;
  static constexpr int TX = 3 * KB * kWin * R;                     // bytes the copies deliver
};

__host__ __device__ constexpr int conv_tma_smem_bytes(int cin, int ns) {
  return 1024 + 3 * (cin < 64 ? 1 : cin / 64) * ((kWin * (cin < 64 ? cin * 2 : 128) + 1023) / 1024) * 1024 +
         9 * cin * ns * 2;
}
constexpr int kConvSmemMax = 200 * 1024;
// the widest output slice that fits (COUT itself when it does)
__host__ __device__ constexpr int conv_ns_wide(int cin, int cout) {
  return conv_tma_smem_bytes(cin, cout) <= kConvSmemMax ? cout : 32;
}

template <int CIN, int COUT, int NS>
__global__ void __launch_bounds__(128) conv3x3_tma_kernel(const __grid_constant__ CUtensorMap tmap, ConvArgs a) {
  using namespace tpf::tc;
  using G = WinGeom<CIN>;
  constexpr int KCH = CIN / 8;
  constexpr int WBYTES = 9 * CIN * NS * 2;
  constexpr int NCOLS = NS < 32 ? 32 : NS;
  constexpr uint32_t IDESC = idesc_bf16_f32(kTile, NS);
  static_assert(CIN % 16 == 0 && COUT % NS == 0 && NS % 16 == 0 && NS <= 256, "conv shape");
  static_assert(conv_tma_smem_bytes(CIN, NS) <= kConvSmemMax, "conv shared memory");

  extern __shared__ unsigned char smem_raw[];
  __shared__ uint64_t lbar, mbar;
  __shared__ uint32_t tmem_slot;
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char* sA = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  unsigned char* sB = sA + G::BYTES;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long q0 = (long long)blockIdx.x * kTile;
  const int n0 = blockIdx.y * NS;

  pdl_trigger();   // the next layer may start its prologue
  if (warp == 0) tmem_alloc(&tmem_slot, NCOLS);
  if (tid == 0) {
    mbar_init(&lbar, 1);
    mbar_init(&mbar, 1);
    mbar_fence_init();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;

  // the weights do not depend on the previous layer: request them before waiting for it
  if (warp == 0) {
    if (lane == 0) mbar_arrive_expect_tx(&lbar, WBYTES + G::TX);
    __syncwarp();
    const unsigned char* wsrc = reinterpret_cast<const unsigned char*>(a.w);
    if (NS == COUT) {
      if (lane == 0) bulk_load(sB, wsrc, WBYTES, &lbar);
    } else {
      for (int pl = lane; pl < 9 * KCH; pl += 32)
        bulk_load(sB + pl * NS * 16, wsrc + ((size_t)pl * COUT + n0) * 16, NS * 16, &lbar);
    }
  }
  pdl_wait();
  if (tid == 0) {
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      const int y = (int)(q0 - 1 + (long long)(w - 1) * a.Wp);
#pragma unroll
      for (int kb = 0; kb < G::KB; ++kb) tensor_load_2d(sA + (w * G::KB + kb) * G::BLOCK, &tmap, kb * 64, y, &lbar);
    }
  }

  bool ok = true;
  if (tid == 0) {
    if (!mbar_wait(&lbar, 0, kSpin)) {
      ok = false;
      mbar_wait(&lbar, 0, kSpin);   // let copies still in flight land before going on
    }
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
      const int dy = tap / 3, dx = tap - (tap / 3) * 3;   // 0..2
#pragma unroll
      for (int kc = 0; kc < CIN / 16; ++kc) {
        const int kb = (kc * 32) / G::R, koff = (kc * 32) % G::R;
        const uint64_t ad = smem_desc_swizzled(a0 + (dy * G::KB + kb) * G::BLOCK + dx * G::R + koff, G::R);
        const uint64_t bd = smem_desc(b0 + (tap * KCH + 2 * kc) * (NS * 16), NS * 16, 128);
        mma_bf16(tmem, ad, bd, IDESC, (tap > 0 || kc > 0) ? 1u : 0u);
      }
    }
    mma_commit(&mbar);
  }
  __syncwarp();
  if (!mbar_wait(&mbar, 0, kSpin)) ok = false;
  fence_after_sync();
  if (!ok) atomicExch(a.err, 1);

  // epilogue: warp w owns TMEM lanes / tile pixels [32w, 32w + 32)
  const long long q = q0 + warp * 32 + lane;
  const bool inb = q < a.P;
  const bool inner = inb && interior_pixel(q, a.Hp, a.Wp);
#pragma unroll 1
  for (int c0 = 0; c0 < NS; c0 += 16) {
    float v[16];
    tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
    if (inb) {
      const int co = n0 + c0;
      float m[16];
      if (a.mask && inner) {
        const uint4* mp = reinterpret_cast<const uint4*>(a.mask + q * COUT + co);
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
        if (a.bias) { x0 += a.bias[co + i]; x1 += a.bias[co + i + 1]; }
        if (a.relu) { x0 = fmaxf(x0, 0.f); x1 = fmaxf(x1, 0.f); }
        x0 *= m[i];
        x1 *= m[i + 1];
        if (!inner) { x0 = 0.f; x1 = 0.f; }
        o2[i / 2] = __floats2bfloat162_rn(x0, x1);
      }
      uint4* op = reinterpret_cast<uint4*>(a.out + q * COUT + co);
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

// Per-item bodies of the resampling layers, shared by the standalone kernels
// and the persistent forward.  Inputs are read through L2 (ld.global.cg):
// inside the persistent forward they were written by other SMs in an
// earlier stage of the same launch.

// out(level l+1) = 2x2 average of in(level l); item i = (pixel, 8-channel group)
template <int C>
__device__ __forceinline__ void pool_item(const LevelGeom& gi, const LevelGeom& go, const bf16* in, bf16* out,
                                          long long i) {
  constexpr int K = C / 8;
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
        unpack8(__ldcg(reinterpret_cast<const uint4*>(in + gi.q(b, 2 * y + dy, 2 * x + dx) * C) + c), f);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += 0.25f * f[k];
      }
  }
  reinterpret_cast<uint4*>(out + q * C)[c] = pack8(acc);
}

// out(level l) = relu(up(t)(level l+1 -> l) + skip)
template <int C>
__device__ __forceinline__ void upadd_item(const LevelGeom& gf, const LevelGeom& gc, const bf16* t, const bf16* skip,
                                           bf16* out, long long i) {
  constexpr int K = C / 8;
  const long long q = i / K;
  const int c = (int)(i - q * K);
  int b, y, x;
  float o[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (pix(gf, q, b, y, x)) {
    float f[8], s[8];
    unpack8(__ldcg(reinterpret_cast<const uint4*>(t + gc.q(b, y >> 1, x >> 1) * C) + c), f);
    unpack8(__ldcg(reinterpret_cast<const uint4*>(skip + q * C) + c), s);
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = fmaxf(f[k] + s[k], 0.f);
  }
  reinterpret_cast<uint4*>(out + q * C)[c] = pack8(o);
}

// y = d0 . w_out + b_out for the 16 channels of one pixel
__device__ __forceinline__ float out1x1_value(const uint4& lo, const uint4& hi, const float* w, const float* bo) {
  float f[8], acc = *bo;
  unpack8(lo, f);
#pragma unroll
  for (int k = 0; k < 8; ++k) acc += f[k] * w[k];
  unpack8(hi, f);
#pragma unroll
  for (int k = 0; k < 8; ++k) acc += f[k] * w[8 + k];
  return acc;
}

template <int C>
__global__ void pool_kernel(LevelGeom gi, LevelGeom go, const bf16* in, bf16* out) {
  tpf::chain_begin();
  tpf::tc::pdl_trigger();
  const long long n = go.P() * (C / 8);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    pool_item<C>(gi, go, in, out, i);
  tpf::chain_end();
}

template <int C>
__global__ void upadd_relu_kernel(LevelGeom gf, LevelGeom gc, const bf16* t, const bf16* skip, bf16* out) {
  tpf::chain_begin();
  tpf::tc::pdl_trigger();
  const long long n = gf.P() * (C / 8);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    upadd_item<C>(gf, gc, t, skip, out, i);
  tpf::chain_end();
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
  tpf::chain_begin();
  const long long n = (long long)g.B * g.H * g.W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.W);
    const long long t = i / g.W;
    const int y = (int)(t % g.H);
    const int b = (int)(t / g.H);
    const uint4* p = reinterpret_cast<const uint4*>(d0 + g.q(b, y, x) * kOutC);
    yout[i] = out1x1_value(p[0], p[1], w, bo);
  }
  tpf::chain_end();
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

// ---- persistent forward ---------------------------------------------------------------------
// The whole forward pass in ONE cooperative launch (one 128-thread CTA per
// SM): 14 convolution stages, 3 poolings and 3 upsample-adds separated by
// grid barriers, the 1x1 output fused into the last convolution's epilogue.
// TMEM is held for the whole launch, the next convolution's weights are
// fetched before the barrier that precedes it, and the deep (few-tile) layers
// split their output channels over CTAs (N = nc per MMA) so that more SMs
// share them.  Every output element sees the same MMA sequence (taps, then
// 16-channel K steps) as in the layered kernel, so the outputs are identical.
// Measured at the preconditioner's 136^2 image (batch 1): ~106 us inside the
// kernel, of which ~19 us are the 19 barriers; the largest part of a stage is
// gathering the 16-byte channel chunks of the three input windows out of the
// pixel-major activations (~29 GB/s per SM, against ~150 GB/s for a linear
// copy), then the MMA issue (~37 ns per M128 x N16 x K16 instruction).
constexpr int kPfThreads = 128;
constexpr int kPfCols = 128;                         // TMEM columns held (max nc)
constexpr int kPfWin = 3 * (128 / 8) * kPlane;       // windows of a 128-channel input
constexpr int kPfW = 9 * 128 * 32 * 2;               // weights of one unit (max 9 * cin * nc * 2)
constexpr int kPfBias = 128 * 4;                     // biases of one unit (max nc floats)
constexpr int kPfSmem = kPfWin + kPfW + kPfBias;

struct PfConv {
  const bf16* in;     // [P][cin]
  bf16* out;          // [P][cout]
  const bf16* w;      // [9][cin/8][cout][8]
  const float* bias;  // [cout]
  long long P;
  int Hp, Wp, cin, cout, nc, tiles, relu;
};
struct PfArgs {
  PfConv c[kConvs];
  LevelGeom g[4];
  const bf16 *e0, *e1, *e2, *t2, *t1, *t0;
  bf16 *p0, *p1, *p2, *d2a, *d1a, *d0a;
  const float* w_out;
  const float* b_out;
  float* y;                  // [B][H][W]
  unsigned long long* bar;   // monotonic arrival counter of the grid barriers
  int* err;
};
struct PfCtx {
  int wl, wc;          // layer / channel chunk whose weights are in (or on the way to) shared memory
  uint32_t phase, tmem;
  bool ok;
};

__device__ __forceinline__ unsigned long long pf_ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void pf_red_release_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}

// Grid barrier on a monotonic 64-bit arrival counter: one release-add per CTA
// and acquire polling, no reset.  Every launch adds exactly kPfBarriers x
// gridDim.x arrivals (a CTA whose wait gives up still arrives at every later
// barrier), so a launch finds its base as the counter rounded down to that
// multiple: before barrier 0 completes the counter is at most
// base + gridDim.x - 1.  Bounded wait; gives up (error flag) rather than hang.
constexpr int kPfBarriers = 19;
struct PfBarrier {
  unsigned long long* count;
  unsigned long long target;   // arrivals that complete the next barrier
};
__device__ __forceinline__ PfBarrier pf_barrier_begin(unsigned long long* count) {
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) {
    const unsigned long long c = pf_ld_acquire(count);
    const unsigned long long per = (unsigned long long)kPfBarriers * gridDim.x;
    s_base = c - c % per;
  }
  __syncthreads();
  return PfBarrier{count, s_base + gridDim.x};
}
__device__ __forceinline__ void pf_grid_sync(PfBarrier& br, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    pf_red_release_add(br.count, 1ull);
    long long spins = 0;
    while (pf_ld_acquire(br.count) < br.target) {
      if (++spins > kSpin) { atomicExch(err, 1); break; }
      if ((spins & 255) == 0 && *(volatile int*)err) break;
    }
  }
  br.target += gridDim.x;
  __syncthreads();
}

// weights of output channels [chunk*nc, (chunk+1)*nc) -> smem [9][cin/8][nc][8],
// followed (at kPfW) by their nc biases (the bias offsets of the flat
// parameter layout are multiples of 16 floats, so the copy is 16-byte
// aligned).  Consecutive threads copy consecutive 16-byte pieces on both sides.
__device__ __forceinline__ void pf_load_weights(const PfConv& L, int chunk, unsigned char* sB) {
  const int lg = L.nc == 16 ? 4 : (L.nc == 32 ? 5 : (L.nc == 64 ? 6 : 7));   // nc is a power of two
  const int n = 9 * (L.cin / 8) << lg;      // 16-byte pieces: (tap, 8-channel) rows x nc
  const unsigned char* src = reinterpret_cast<const unsigned char*>(L.w);
  for (int i = threadIdx.x; i < n; i += kPfThreads) {
    const int r = i >> lg, j = i & (L.nc - 1);
    tpf::tc::cp_async16(sB + (size_t)i * 16, src + ((size_t)r * L.cout + (size_t)chunk * L.nc + j) * 16, true);
  }
  if ((int)threadIdx.x < L.nc / 4)
    tpf::tc::cp_async16(sB + kPfW + threadIdx.x * 16, L.bias + (size_t)chunk * L.nc + threadIdx.x * 4, true);
  tpf::tc::cp_async_commit();
}

// fetch the weights of this CTA's first unit of layer l (if it has one)
__device__ __forceinline__ void pf_prefetch(const PfArgs& a, int l, PfCtx& cx, unsigned char* sB) {
  if (l >= kConvs) return;
  const PfConv& L = a.c[l];
  if ((int)blockIdx.x >= L.tiles * (L.cout / L.nc)) return;
  const int chunk = (int)blockIdx.x / L.tiles;
  pf_load_weights(L, chunk, sB);
  cx.wl = l;
  cx.wc = chunk;
}

// One convolution stage.  Per unit (128 output pixels x nc output channels):
// the three windows (and, unless prefetched, the weight chunk) are copied
// into shared memory, thread 0 issues 9 x CIN/16 tcgen05.mma (M = 128,
// N = nc, K = 16) with descriptors advanced by constant offsets, and four
// warps read TMEM back for the bias / ReLU / border epilogue.  CIN is a
// compile-time constant so that the addressing divides by constants and the
// MMA issue is straight-line code.
template <int CIN>
__device__ void pf_conv_t(const PfArgs& a, int l, PfCtx& cx, unsigned char* smem, uint64_t* mbar) {
  using namespace tpf::tc;
  constexpr int WIN_BYTES = (CIN / 8) * kPlane;
  const PfConv& L = a.c[l];
  const int units = L.tiles * (L.cout / L.nc);
  unsigned char* sA = smem;
  unsigned char* sB = smem + kPfWin;
  const float* sBias = reinterpret_cast<const float*>(sB + kPfW);
  if ((int)blockIdx.x >= units) {
    pf_prefetch(a, l + 1, cx, sB);
    return;
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nc = L.nc;
  const uint32_t idesc = idesc_bf16_f32(kTile, nc);
  for (int u = blockIdx.x; u < units; u += gridDim.x) {
    const int chunk = u / L.tiles;
    const long long q0 = (long long)(u - chunk * L.tiles) * kTile;
    if (cx.wl != l || cx.wc != chunk) {
      pf_load_weights(L, chunk, sB);
      cx.wl = l;
      cx.wc = chunk;
    }
    load_windows<CIN>(L.in, L.P, L.Wp, q0, sA);
    cp_async_wait_all();
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      // descriptor address fields are in 16-byte units; every offset below
      // keeps the address inside shared memory, so adding to the low field
      // never carries into the next one
      const uint64_t ad0 = smem_desc(smem_u32(sA), kPlane, 128);
      const uint64_t bd0 = smem_desc(smem_u32(sB), nc * 16, 128);
      const uint32_t tap_step = (uint32_t)(CIN * nc * 2) >> 4, kc_step = (uint32_t)(nc * 32) >> 4;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap % 3;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; ++kc) {
          const uint64_t ad = ad0 + (uint64_t)((dy * WIN_BYTES + dx * 16 + kc * 2 * kPlane) >> 4);
          const uint64_t bd = bd0 + (uint64_t)(tap * tap_step + kc * kc_step);
          mma_bf16(cx.tmem, ad, bd, idesc, (tap > 0 || kc > 0) ? 1u : 0u);
        }
      }
      mma_commit(mbar);
    }
    __syncwarp();
    if (!mbar_wait(mbar, cx.phase, kSpin)) cx.ok = false;
    cx.phase ^= 1u;
    fence_after_sync();
    const long long q = q0 + warp * 32 + lane;
    const bool inb = q < L.P;
    const bool inner = inb && interior_pixel(q, L.Hp, L.Wp);
    const int n0 = chunk * nc;
    const bool last_unit = u + (int)gridDim.x >= units;
#pragma unroll 1
    for (int c0 = 0; c0 < nc; c0 += 16) {
      float v[16], bv[16];
      tmem_ld16(cx.tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) bv[i] = sBias[c0 + i];
      if (inb) {
        uint4 ov[2];
        __nv_bfloat162* o2 = reinterpret_cast<__nv_bfloat162*>(ov);
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
          float x0 = v[i] + bv[i], x1 = v[i + 1] + bv[i + 1];
          if (L.relu) { x0 = fmaxf(x0, 0.f); x1 = fmaxf(x1, 0.f); }
          if (!inner) { x0 = 0.f; x1 = 0.f; }
          o2[i / 2] = __floats2bfloat162_rn(x0, x1);
        }
        uint4* op = reinterpret_cast<uint4*>(L.out + q * L.cout + n0 + c0);
        op[0] = ov[0];
        op[1] = ov[1];
        if (l == kConvs - 1 && inner) {   // fused 1x1 output (cout == nc == 16)
          int b, yy, xx;
          pix(a.g[0], q, b, yy, xx);
          a.y[((long long)b * a.g[0].H + yy) * a.g[0].W + xx] = out1x1_value(ov[0], ov[1], a.w_out, a.b_out);
        }
      }
    }
    fence_before_sync();
    __syncthreads();
    // windows, weights and biases are consumed: the next layer's weights can
    // stream in during the barrier that follows
    if (last_unit) pf_prefetch(a, l + 1, cx, sB);
  }
}

__device__ __forceinline__ void pf_conv(const PfArgs& a, int l, PfCtx& cx, unsigned char* smem, uint64_t* mbar) {
  switch (a.c[l].cin) {
    case 16: pf_conv_t<16>(a, l, cx, smem, mbar); break;
    case 32: pf_conv_t<32>(a, l, cx, smem, mbar); break;
    case 64: pf_conv_t<64>(a, l, cx, smem, mbar); break;
    default: pf_conv_t<128>(a, l, cx, smem, mbar); break;
  }
}

template <int C>
__device__ __forceinline__ void pf_pool(const LevelGeom& gi, const LevelGeom& go, const bf16* in, bf16* out) {
  const long long n = go.P() * (C / 8);
  for (long long i = blockIdx.x * (long long)kPfThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kPfThreads)
    pool_item<C>(gi, go, in, out, i);
}
template <int C>
__device__ __forceinline__ void pf_upadd(const LevelGeom& gf, const LevelGeom& gc, const bf16* t, const bf16* skip,
                                         bf16* out) {
  const long long n = gf.P() * (C / 8);
  for (long long i = blockIdx.x * (long long)kPfThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kPfThreads)
    upadd_item<C>(gf, gc, t, skip, out, i);
}

__global__ void __launch_bounds__(kPfThreads, 1) unet_forward_persistent_kernel(const __grid_constant__ PfArgs a) {
  using namespace tpf::tc;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) tmem_alloc(&tmem_slot, kPfCols);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_fence_init();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  PfCtx cx{-1, -1, 0u, tmem_slot, true};
  pf_prefetch(a, 0, cx, smem + kPfWin);
  PfBarrier br = pf_barrier_begin(a.bar);

  pf_conv(a, 0, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 1, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_pool<16>(a.g[0], a.g[1], a.e0, a.p0);
  pf_grid_sync(br, a.err);
  pf_conv(a, 2, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 3, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_pool<32>(a.g[1], a.g[2], a.e1, a.p1);
  pf_grid_sync(br, a.err);
  pf_conv(a, 4, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 5, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_pool<64>(a.g[2], a.g[3], a.e2, a.p2);
  pf_grid_sync(br, a.err);
  pf_conv(a, 6, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 7, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 8, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_upadd<64>(a.g[2], a.g[3], a.t2, a.e2, a.d2a);
  pf_grid_sync(br, a.err);
  pf_conv(a, 9, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 10, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_upadd<32>(a.g[1], a.g[2], a.t1, a.e1, a.d1a);
  pf_grid_sync(br, a.err);
  pf_conv(a, 11, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_conv(a, 12, cx, smem, &mbar);
  pf_grid_sync(br, a.err);
  pf_upadd<16>(a.g[0], a.g[1], a.t0, a.e0, a.d0a);
  pf_grid_sync(br, a.err);
  pf_conv(a, 13, cx, smem, &mbar);

  if (!cx.ok) atomicExch(a.err, 1);
  // a CTA without units in the last layers may still have a weight copy in flight
  cp_async_wait_all();
  fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(cx.tmem, kPfCols);
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
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

// Tensor map of the pixel-major [P][CIN] BF16 activations read by the
// convolution: boxes of 130 pixels x min(CIN, 64) channels, swizzled to match
// the MMA operand layout.
int window_map(CUtensorMap* m, const bf16* in, int cin, long long P) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) {
    tpf::set_error("cuTensorMapEncodeTiled is not available from the driver");
    return TPF_ECUDA;
  }
  const int box_c = cin < 64 ? cin : 64;
  const cuuint64_t dims[2] = {(cuuint64_t)cin, (cuuint64_t)P};
  const cuuint64_t strides[1] = {(cuuint64_t)cin * sizeof(bf16)};
  const cuuint32_t box[2] = {(cuuint32_t)box_c, (cuuint32_t)kWin};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapSwizzle sw = box_c == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                            : (box_c == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(in), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    tpf::set_error("cuTensorMapEncodeTiled failed (%d) for %d channels x %lld pixels", (int)r, cin, P);
    return TPF_ECUDA;
  }
  return TPF_OK;
}

template <int CIN, int COUT, int NS>
int launch_conv_ns(const CUtensorMap& m, const ConvArgs& a, long long tiles, cudaStream_t s) {
  constexpr int smem = conv_tma_smem_bytes(CIN, NS);
  static bool attr = false;
  if (!attr) {
    TPF_CUDA_TRY(cudaFuncSetAttribute(conv3x3_tma_kernel<CIN, COUT, NS>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  // programmatic dependent launch: the prologue overlaps the previous kernel,
  // whose outputs are read only after griddepcontrol.wait
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)tiles, COUT / NS);
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl;
  cfg.numAttrs = 1;
  TPF_CUDA_TRY(cudaLaunchKernelEx(&cfg, conv3x3_tma_kernel<CIN, COUT, NS>, m, a));
  return TPF_OK;
}

// Output slices: the whole COUT per CTA when the pixel tiles alone fill the
// GPU, else 16 channels per CTA (more CTAs, each with less weight traffic).
template <int CIN, int COUT>
int launch_conv_t(const ConvArgs& a, cudaStream_t s) {
  CUtensorMap m;
  int st = window_map(&m, a.in, CIN, a.P);
  if (st) return st;
  const long long tiles = (a.P + kTile - 1) / kTile;
  constexpr int NW = conv_ns_wide(CIN, COUT);
  if (tiles >= 128 || COUT == 16) return launch_conv_ns<CIN, COUT, NW>(m, a, tiles, s);
  return launch_conv_ns<CIN, COUT, 16>(m, a, tiles, s);
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
  unsigned long long* bar = nullptr;   // grid-barrier counter of the persistent forward
  int forward_mode = 0;                // 0 layered launches, 1 persistent launch
  PfArgs* pf_args = nullptr;           // launch arguments of the persistent forward
  int pf_batch = 0;                    // ... built for this batch size (0: none)
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
  tpf::launch_chained(pool_kernel<C>, grid_for(go.P() * (C / 8)), 256, 0, s, gi, go, in, out);
}
template <int C>
void upadd_t(const LevelGeom& gf, const LevelGeom& gc, const bf16* t, const bf16* sk, bf16* out, cudaStream_t s) {
  tpf::launch_chained(upadd_relu_kernel<C>, grid_for(gf.P() * (C / 8)), 256, 0, s, gf, gc, t, sk, out);
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

// CTAs of the persistent forward: one per SM (cooperative launch)
int persistent_grid() {
  static int grid = -1;
  if (grid < 0) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(unet_forward_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kPfSmem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, unet_forward_persistent_kernel, kPfThreads,
                                                      kPfSmem) != cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      grid = 0;
    } else {
      grid = sms;
    }
  }
  return grid;
}

// output-channel split of a convolution in the persistent forward: as many
// 16-channel chunks as keep units (tiles x chunks) within one wave, and at
// most 32 (128-channel input) or 64 channels per unit (shared-memory bound)
int persistent_nc(int cin, int cout, long long tiles, int grid) {
  const int cap = cin >= 128 ? 32 : 64;
  int split = 1;
  while (cout / split > cap) split *= 2;
  while (cout / (split * 2) >= 16 && tiles * split * 2 <= grid) split *= 2;
  return cout / split;
}

// launch arguments of the persistent forward for batch B (the channel
// splits depend only on B, the addresses are fixed per workspace)
int build_persistent_args(tpf_unet* n, int B, int grid, PfArgs& a) {
  const ParamLayout& L = layout();
  a = PfArgs{};
  const bf16* ins[kConvs] = {n->xin, n->e0a, n->p0, n->e1a, n->p1, n->e2a, n->p2,
                             n->e3a, n->e3,  n->d2a, n->d2, n->d1a, n->d1, n->d0a};
  bf16* outs[kConvs] = {n->e0a, n->e0, n->e1a, n->e1, n->e2a, n->e2, n->e3a,
                        n->e3,  n->t2, n->d2,  n->t1, n->d1,  n->t0, n->d0};
  for (int l = 0; l < kConvs; ++l) {
    const LevelGeom g = n->geom(kLayers[l].level, B);
    PfConv& c = a.c[l];
    c.in = ins[l];
    c.out = outs[l];
    c.w = n->wf[l];
    c.bias = n->params + L.b[l];
    c.P = g.P();
    c.Hp = g.Hp;
    c.Wp = g.Wp;
    c.cin = cin_kernel(l);
    c.cout = kLayers[l].cout;
    c.relu = kLayers[l].relu;
    const long long tiles = (c.P + kTile - 1) / kTile;
    c.tiles = (int)tiles;
    c.nc = persistent_nc(c.cin, c.cout, tiles, grid);
  }
  for (int l = 0; l < 4; ++l) a.g[l] = n->geom(l, B);
  a.e0 = n->e0;
  a.e1 = n->e1;
  a.e2 = n->e2;
  a.t2 = n->t2;
  a.t1 = n->t1;
  a.t0 = n->t0;
  a.p0 = n->p0;
  a.p1 = n->p1;
  a.p2 = n->p2;
  a.d2a = n->d2a;
  a.d1a = n->d1a;
  a.d0a = n->d0a;
  a.w_out = n->params + L.wo;
  a.b_out = n->params + L.bo;
  a.y = n->out;
  a.bar = n->bar;
  a.err = n->err;
  return TPF_OK;
}

int forward_persistent(tpf_unet* n, int B, cudaStream_t s) {
  const int grid = persistent_grid();
  if (grid <= 0) {
    tpf::set_error("the persistent forward cannot be made co-resident on this device");
    return TPF_ECUDA;
  }
  if (!n->pf_args) n->pf_args = new PfArgs();
  if (n->pf_batch != B) {
    n->pf_batch = 0;
    int st = build_persistent_args(n, B, grid, *n->pf_args);
    if (st) return st;
    n->pf_batch = B;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kPfThreads);
  cfg.dynamicSmemBytes = kPfSmem;
  cfg.stream = s;
  cudaLaunchAttribute coop[1];
  coop[0].id = cudaLaunchAttributeCooperative;
  coop[0].val.cooperative = 1;
  cfg.attrs = coop;
  cfg.numAttrs = 1;
  TPF_CUDA_TRY(cudaLaunchKernelEx(&cfg, unet_forward_persistent_kernel, *n->pf_args));
  return TPF_OK;
}

// The layered launches are the default: inside the learned solver's CUDA
// graph they overlap their prologues with the previous kernel (programmatic
// dependent launch), which the cooperative launch cannot, and measured
// faster there (161 vs 187 us per flexible-CG iteration at 512^2); the
// persistent launch is faster for a stand-alone forward call.
bool use_persistent(const tpf_unet* n, int) { return n->forward_mode == 1; }

int forward(tpf_unet* n, int B, cudaStream_t s) {
  int st;
  if (!n->arranged && (st = arrange(n, s))) return st;
  if (use_persistent(n, B)) {
    if ((st = forward_persistent(n, B, s))) return st;
    n->last_batch = B;
    return TPF_OK;
  }

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
  tpf::launch_chained(out1x1_kernel, grid_for((long long)B * n->H * n->W), 256, 0, s, g0, n->d0, n->params + L.wo,
                      n->params + L.bo, n->out);
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
    // start the next call clean: a timed-out wait leaves the flag set
    cudaMemsetAsync(n->bar, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(n->err, 0, sizeof(int), s);
    cudaStreamSynchronize(s);
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
  if ((st = ualloc(n, &n->bar, 1))) return fail(st);
  TPF_CUDA_TRY(cudaMemset(n->bar, 0, sizeof(unsigned long long)));
  *out = n;
  return TPF_OK;
}

int tpf_unet_destroy(tpf_unet* n) {
  if (!n) return TPF_OK;
  cudaDeviceSynchronize();
  for (void* p : n->allocs) cudaFree(p);
  delete n->pf_args;
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

int tpf_unet_set_forward_mode(tpf_unet* n, int mode) {
  TPF_CHECK_ARG(n != nullptr, "null handle");
  TPF_CHECK_ARG(mode >= -1 && mode <= 1, "forward mode must be -1, 0 or 1 (got %d)", mode);
  n->forward_mode = mode < 0 ? 0 : mode;
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

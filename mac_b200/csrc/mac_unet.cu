// Learned preconditioner: a 3-level 3D U-Net (16/32/64 channels, 3x3x3
// convolutions, ReLU, BF16 weights and activations, FP32 accumulation) run as
// implicit-GEMM convolutions on the tcgen05 tensor cores, with hand-written
// forward, backward (input and weight gradients) and Adam kernels, and the
// generator of its training pairs (residual, exact error) from plain FP64 CG
// iterates on random fluid masks.
//
// No counterpart in the reference (its solvers are Umfpack and pyamg:
// src/Policy_Solve_Linear_Umfpack.h, src/Algorithms_Solve_Pressure_Pyamg.h).
//
// Layout: activations are channels-last [n][z][y][x][c] BF16 with c a multiple
// of 16; weights are [tap][cout][cin] (tap = 9 (dz+1) + 3 (dy+1) + (dx+1)).
// A convolution is the GEMM  out[voxel][co] = sum_{tap, ci} in[voxel + off(tap)][ci] * W[tap][co][ci]
// with M = 128 output voxels per CTA, N = output channels, K = input channels
// per tap; both operands are gathered with plain 16-byte copies (a voxel's 8
// channels are one row of a core matrix), and the accumulator lives in tensor
// memory. The input gradient is the same GEMM with negated tap offsets and the
// weights read MN-major; the weight gradient contracts over voxels with both
// operands MN-major and a split-K FP32 atomic reduction.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mac_internal.cuh"
#include "mac_unet.cuh"
#include "mac_unet_mma.cuh"

namespace mac {
namespace unet {

using bf16 = __nv_bfloat16;

// ------------------------------------------------------------------ network
const LayerDef kLayers[kNumLayers] = {
    // cin, cout, taps, relu, real_cin, real_cout
    {16, 16, 27, 1, 2, 16},   // 0 enc1a (input channels: residual, mask)
    {16, 16, 27, 1, 16, 16},  // 1 enc1b -> skip 1
    {16, 32, 27, 1, 16, 32},  // 2 enc2a (after 2x average pool)
    {32, 32, 27, 1, 32, 32},  // 3 enc2b -> skip 2
    {32, 64, 27, 1, 32, 64},  // 4 enc3a (after 2x average pool)
    {64, 64, 27, 1, 64, 64},  // 5 enc3b
    {64, 32, 1, 0, 64, 32},   // 6 up2: 1x1 at the coarse level, read 2x upsampled by dec2a
    {64, 32, 27, 1, 64, 32},  // 7 dec2a on concat(skip 2, up2)
    {32, 32, 27, 1, 32, 32},  // 8 dec2b
    {32, 16, 1, 0, 32, 16},   // 9 up1: 1x1, read 2x upsampled by dec1a
    {32, 16, 27, 1, 32, 16},  // 10 dec1a on concat(skip 1, up1)
    {16, 16, 27, 1, 16, 16},  // 11 dec1b
    {16, 16, 1, 0, 16, 1},    // 12 output: 1x1, channel 0 only
};

// Activation tensors: channels and level (0 = full grid, 1 = half, 2 = quarter).
const int kActCh[kNumAct] = {16, 16, 16, 16, 32, 32, 32, 64, 64, 32, 32, 32, 16, 16, 16, 16, 32, 16};
const int kActLvl[kNumAct] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 2, 1, 1, 1, 0, 0, 0, 1, 0};

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ uint4 ldg16(const bf16* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

// Keeps each BF16 lane of g where the matching lane of y is > 0 (ReLU backward).
__device__ __forceinline__ uint32_t gate2(uint32_t g, uint32_t y) {
  uint32_t lo = y & 0xFFFFu, hi = y >> 16;
  uint32_t mlo = (lo != 0 && !(lo & 0x8000u)) ? 0xFFFFu : 0u;
  uint32_t mhi = (hi != 0 && !(hi & 0x8000u)) ? 0xFFFF0000u : 0u;
  return g & (mlo | mhi);
}
__device__ __forceinline__ uint4 gate8(uint4 g, uint4 y) {
  return make_uint4(gate2(g.x, y.x), gate2(g.y, y.y), gate2(g.z, y.z), gate2(g.w, y.w));
}

// 8 channels (16 bytes) starting at channel 8*chunk of concat(s1, s2) at the
// full-resolution voxel (n, z, y, x) of a d x h x w grid; s2 may be stored at
// half resolution (nearest upsampling).
__device__ __forceinline__ uint4 gather8(const Src& s1, const Src& s2, int chunk, int n, int z, int y, int x,
                                         int d, int h, int w) {
  int ch = chunk * 8;
  const bool first = ch < s1.c;
  const bf16* p = first ? s1.p : s2.p;
  int c = first ? s1.c : s2.c;
  int sh = first ? s1.shift : s2.shift;
  if (!first) ch -= s1.c;
  size_t v = (((size_t)n * (d >> sh) + (z >> sh)) * (h >> sh) + (y >> sh)) * (w >> sh) + (x >> sh);
  return ldg16(p + v * c + ch);
}

__device__ __forceinline__ void tap_offset(int t, int taps, int& dz, int& dy, int& dx) {
  if (taps == 27) {
    dz = t / 9 - 1;
    dy = (t / 3) % 3 - 1;
    dx = t % 3 - 1;
  } else {
    dz = dy = dx = 0;
  }
}

// Sum over a block of up to 1024 threads; the result is valid in thread 0.
__device__ inline double bsum(double a) {
  __shared__ double red[32];
  for (int s = 16; s > 0; s >>= 1) a += __shfl_down_sync(0xffffffffu, a, s);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// ------------------------------------------------------- convolution (M = voxels)
// MODE 0: forward, out = act(conv(in) + bias), B = W K-major.
// MODE 1: input gradient, out = conv(g * gate) with negated taps, B = W MN-major;
//         output channels [0, c1) go to d1 and [c1, NC) to d2.
constexpr int kConvStages = 4;

template <int KC, int NC>
constexpr int conv_smem() {
  return kConvStages * (128 * KC * 2 + NC * KC * 2) + 128;
}

template <int KC, int NC, int MODE>
__global__ void __launch_bounds__(128) k_conv(ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int A_BYTES = 128 * KC * 2;
  constexpr int B_BYTES = NC * KC * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr uint32_t SBO = (KC / 8) * 128;
  constexpr uint32_t TCOLS = NC < 32 ? 32 : NC;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, NC, 0, MODE);
  uint64_t* freeb = reinterpret_cast<uint64_t*>(smem + kConvStages * STAGE);
  uint64_t* done = freeb + kConvStages;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < kConvStages; ++s) umma::mbar_init(&freeb[s], 1);
    umma::mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 0) umma::tmem_alloc(tslot, TCOLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;

  const int V = a.n * a.d * a.h * a.w;
  const int v = blockIdx.x * 128 + tid;
  const bool valid = v < V;
  int x = v % a.w, r = v / a.w;
  int y = r % a.h;
  r /= a.h;
  int z = r % a.d, n = r / a.d;

  bool ok = true;
  for (int t = 0; t < a.taps; ++t) {
    const int s = t % kConvStages;
    uint8_t* As = smem + s * STAGE;
    uint8_t* Bs = As + A_BYTES;
    if (t >= kConvStages && !umma::mbar_wait(&freeb[s], ((t / kConvStages) - 1) & 1)) ok = false;
    int dz, dy, dx;
    tap_offset(t, a.taps, dz, dy, dx);
    if (MODE == 1) {
      dz = -dz;
      dy = -dy;
      dx = -dx;
    }
    const int sz = z + dz, sy = y + dy, sx = x + dx;
    const bool inb = valid && sz >= 0 && sz < a.d && sy >= 0 && sy < a.h && sx >= 0 && sx < a.w;
#pragma unroll
    for (int c = 0; c < KC / 8; ++c) {
      uint4 val = make_uint4(0, 0, 0, 0);
      if (inb) {
        val = gather8(a.s1, a.s2, c, n, sz, sy, sx, a.d, a.h, a.w);
        if (MODE == 1 && a.gate) {
          size_t gv = (((size_t)n * a.d + sz) * a.h + sy) * a.w + sx;
          val = gate8(val, ldg16(a.gate + gv * KC + c * 8));
        }
      }
      *reinterpret_cast<uint4*>(As + (tid >> 3) * SBO + c * 128 + (tid & 7) * 16) = val;
    }
    // weights of tap t: global rows of CH chunks; forward rows are output
    // channels (K-major tile), input-gradient rows are K (MN-major tile)
    constexpr int ROWS = MODE ? KC : NC;
    constexpr int CH = MODE ? NC / 8 : KC / 8;
    const bf16* wt = a.wt + (size_t)t * NC * KC;
    for (int i = tid; i < ROWS * CH; i += 128) {
      const int row = i / CH, c = i % CH;
      const uint4 val = ldg16(wt + (size_t)row * CH * 8 + c * 8);
      const uint32_t off = MODE ? (c * SBO + (row >> 3) * 128 + (row & 7) * 16)
                                : ((row >> 3) * SBO + c * 128 + (row & 7) * 16);
      *reinterpret_cast<uint4*>(Bs + off) = val;
    }
    umma::fence_async_smem();
    ok = __syncthreads_and(ok);
    if (!ok) break;
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_addr(As), b0 = umma::smem_addr(Bs);
#pragma unroll
      for (int ks = 0; ks < KC / 16; ++ks)
        umma::mma(tmem, umma::desc(a0 + ks * 256, 128, SBO), umma::desc(b0 + ks * 256, 128, SBO), IDESC,
                  (t > 0 || ks > 0) ? 1u : 0u);
      umma::commit(&freeb[s]);
    }
  }
  if (tid == 0) umma::commit(done);
  const bool fin = umma::mbar_wait(done, 0);
  umma::fence_after_sync();
  if (__syncthreads_and(ok && fin)) {
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < NC; c0 += 16) {
      float f[16];
      umma::tmem_ld16(trow + c0, f);
      if (!valid) continue;
      if (MODE == 0) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          if (a.bias) f[i] += a.bias[c0 + i];
          if (a.relu) f[i] = fmaxf(f[i], 0.0f);
        }
        if (a.f32) {
          if (c0 == 0) a.f32[v] = f[0];
          continue;
        }
      }
      uint4 pk[2];
      uint32_t* w32 = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        __nv_bfloat162 b2 = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
        w32[i] = *reinterpret_cast<uint32_t*>(&b2);
      }
      bf16* dst;
      if (c0 < a.c1)
        dst = a.d1 + (size_t)v * a.c1 + c0;
      else
        dst = a.d2 + (size_t)v * (NC - a.c1) + (c0 - a.c1);
      reinterpret_cast<uint4*>(dst)[0] = pk[0];
      reinterpret_cast<uint4*>(dst)[1] = pk[1];
    }
  } else if (tid == 0) {
    atomicExch(a.err, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, TCOLS);
}

// ------------------------------------- forward 3x3x3 convolution, staged tile
// A CTA computes a tile of 8 (x) x 16 (y) x 1 (z) output voxels (M = 128).
// Its input box with a one-voxel halo, 10 x 18 x 3 voxels x KC channels, is
// gathered from global memory once (concatenation and nearest upsampling of
// the sources folded into the gather, zero outside the grid) into the
// no-swizzle K-major layout [channel group g][z][y][x] x 16 bytes. For tap
// (dz, dy, dx) the A operand is then the same box seen from another start
// address: core matrix j (output row y = j, x = 0..7: eight consecutive
// 16-byte rows) starts at ((g*3 + 1+dz)*18 + 1+dy + j)*10 + 1+dx, so the
// M-adjacent core matrices lie SBO = 160 bytes apart and the K-adjacent ones
// LBO = 8640 bytes apart, and the 27 taps need no further gathering. The
// weights of a chunk of taps are staged K-major beside the box; one thread
// issues every tcgen05.mma of the chunk (taps in order, K in steps of 16)
// into the tensor-memory accumulator and commits to an mbarrier (bounded
// wait); the epilogue is k_conv's (bias, ReLU, BF16 or FP32 store). The
// accumulation visits taps and K steps in k_conv's order.
constexpr int kBoxX = 10, kBoxY = 18, kBoxZ = 3, kBoxVox = kBoxX * kBoxY * kBoxZ;
constexpr int kConvWChunk = 65536;  // bytes of weights staged at a time

template <int KC, int NC>
__host__ __device__ constexpr int tile_taps() {
  return (kConvWChunk / (NC * KC * 2)) < 27 ? (kConvWChunk / (NC * KC * 2)) : 27;
}
template <int KC, int NC>
__host__ __device__ constexpr int tile_smem() {
  return KC * kBoxVox * 2 + tile_taps<KC, NC>() * NC * KC * 2 + 128;
}

template <int KC, int NC>
__global__ void __launch_bounds__(128) k_conv_tile(ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int BOX_BYTES = KC * kBoxVox * 2;
  constexpr int TB = tile_taps<KC, NC>();
  constexpr uint32_t LBO_A = kBoxVox * 16, SBO_A = kBoxX * 16;
  constexpr uint32_t SBO_B = (KC / 8) * 128;
  constexpr uint32_t TCOLS = NC < 32 ? 32 : NC;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, NC, 0, 0);
  uint8_t* box = smem;
  uint8_t* wbuf = smem + BOX_BYTES;
  uint64_t* done = reinterpret_cast<uint64_t*>(wbuf + TB * NC * KC * 2);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tx = (a.w + 7) / 8, ty = (a.h + 15) / 16;
  int bid = blockIdx.x;
  const int x0 = (bid % tx) * 8;
  bid /= tx;
  const int y0 = (bid % ty) * 16;
  bid /= ty;
  const int z0 = bid % a.d, n = bid / a.d;
  if (tid == 0) {
    umma::mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 0) umma::tmem_alloc(tslot, TCOLS);
  // the input box, once
  for (int i = tid; i < (KC / 8) * kBoxVox; i += 128) {
    const int g = i / kBoxVox, vox = i - g * kBoxVox;
    const int bx = vox % kBoxX, by = (vox / kBoxX) % kBoxY, bz = vox / (kBoxX * kBoxY);
    const int x = x0 - 1 + bx, y = y0 - 1 + by, z = z0 - 1 + bz;
    uint4 val = make_uint4(0, 0, 0, 0);
    if (x >= 0 && x < a.w && y >= 0 && y < a.h && z >= 0 && z < a.d)
      val = gather8(a.s1, a.s2, g, n, z, y, x, a.d, a.h, a.w);
    *reinterpret_cast<uint4*>(box + (size_t)i * 16) = val;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;
  bool ok = true;
  int phase = 0;
  for (int t0 = 0; t0 < 27; t0 += TB) {
    const int nt = 27 - t0 < TB ? 27 - t0 : TB;
    // weights of taps t0 .. t0+nt-1: rows = output channels, K-major
    for (int i = tid; i < nt * NC * (KC / 8); i += 128) {
      const int tt = i / (NC * (KC / 8)), rem = i - tt * NC * (KC / 8);
      const int row = rem / (KC / 8), c = rem % (KC / 8);
      const uint4 val = ldg16(a.wt + ((size_t)(t0 + tt) * NC + row) * KC + c * 8);
      *reinterpret_cast<uint4*>(wbuf + (size_t)tt * NC * KC * 2 + (row >> 3) * SBO_B + c * 128 + (row & 7) * 16) =
          val;
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t abase = umma::smem_addr(box), bbase = umma::smem_addr(wbuf);
      for (int tt = 0; tt < nt; ++tt) {
        int dz, dy, dx;
        tap_offset(t0 + tt, 27, dz, dy, dx);
        const uint32_t at = abase + (uint32_t)((((1 + dz) * kBoxY + 1 + dy) * kBoxX + 1 + dx) * 16);
        const uint32_t bt = bbase + (uint32_t)(tt * NC * KC * 2);
#pragma unroll
        for (int ks = 0; ks < KC / 16; ++ks)
          umma::mma(tmem, umma::desc(at + ks * 2 * LBO_A, LBO_A, SBO_A), umma::desc(bt + ks * 256, 128, SBO_B),
                    IDESC, (t0 + tt > 0 || ks > 0) ? 1u : 0u);
      }
      umma::commit(done);
    }
    // the next chunk overwrites the weights only after these MMAs completed
    if (!umma::mbar_wait(done, (uint32_t)(phase & 1))) ok = false;
    ++phase;
    umma::fence_after_sync();
    ok = __syncthreads_and(ok);
    if (!ok) break;
  }
  const int m = tid;  // TMEM lane = tile row: x = m & 7, y = m >> 3
  const int x = x0 + (m & 7), y = y0 + (m >> 3);
  const bool valid = x < a.w && y < a.h;
  const size_t v = (((size_t)n * a.d + z0) * a.h + y) * a.w + x;
  if (ok) {
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < NC; c0 += 16) {
      float f[16];
      umma::tmem_ld16(trow + c0, f);
      if (!valid) continue;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        if (a.bias) f[i] += a.bias[c0 + i];
        if (a.relu) f[i] = fmaxf(f[i], 0.0f);
      }
      if (a.f32) {
        if (c0 == 0) a.f32[v] = f[0];
        continue;
      }
      uint4 pk[2];
      uint32_t* w32 = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        __nv_bfloat162 b2 = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
        w32[i] = *reinterpret_cast<uint32_t*>(&b2);
      }
      bf16* dst;
      if (c0 < a.c1)
        dst = a.d1 + v * a.c1 + c0;
      else
        dst = a.d2 + v * (NC - a.c1) + (c0 - a.c1);
      reinterpret_cast<uint4*>(dst)[0] = pk[0];
      reinterpret_cast<uint4*>(dst)[1] = pk[1];
    }
  } else if (tid == 0) {
    atomicExch(a.err, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, TCOLS);
}

// ------------------------------------------------ weight gradient (K = voxels)
// dW[tap][co][ci] += sum_v in[v + off(tap)][ci] * (g * gate)[v][co]; a CTA owns
// 16 (tap, 8-channel group) row blocks = 128 GEMM rows and a range of voxels.
constexpr int kWgStages = 4;
constexpr int kWgK = 64;  // voxels per stage

template <int CIN, int COUT>
constexpr int wgrad_smem() {
  return kWgStages * (16 * kWgK * 16 + (COUT / 8) * kWgK * 16) + 128;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_wgrad(WgradArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int A_BYTES = 16 * kWgK * 16;
  constexpr int B_BYTES = (COUT / 8) * kWgK * 16;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr uint32_t SBO = (kWgK / 8) * 128;
  constexpr uint32_t TCOLS = COUT < 32 ? 32 : COUT;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, COUT, 1, 1);
  uint64_t* freeb = reinterpret_cast<uint64_t*>(smem + kWgStages * STAGE);
  uint64_t* done = freeb + kWgStages;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < kWgStages; ++s) umma::mbar_init(&freeb[s], 1);
    umma::mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 0) umma::tmem_alloc(tslot, TCOLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *tslot;

  const int V = a.n * a.d * a.h * a.w;
  const int mchunks = a.taps * (CIN / 8);
  const int v0 = blockIdx.y * a.vox_per_cta;
  const int v1 = min(V, v0 + a.vox_per_cta);
  const int nst = v0 < v1 ? (v1 - v0 + kWgK - 1) / kWgK : 0;
  const int kk = tid & (kWgK - 1);  // this thread's voxel within a stage
  bool ok = true;
  for (int st = 0; st < nst; ++st) {
    const int s = st % kWgStages;
    uint8_t* As = smem + s * STAGE;
    uint8_t* Bs = As + A_BYTES;
    if (st >= kWgStages && !umma::mbar_wait(&freeb[s], ((st / kWgStages) - 1) & 1)) ok = false;
    const int v = v0 + st * kWgK + kk;
    const bool valid = v < v1;
    int x = v % a.w, r = v / a.w;
    int y = r % a.h;
    r /= a.h;
    int z = r % a.d, n = r / a.d;
    const uint32_t row_off = (kk >> 3) * 128 + (kk & 7) * 16;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int j16 = (tid >> 6) + 2 * j;  // row block (m chunk) within the tile
      const int mc = blockIdx.x * 16 + j16;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (valid && mc < mchunks) {
        const int tap = mc / (CIN / 8), grp = mc % (CIN / 8);
        int dz, dy, dx;
        tap_offset(tap, a.taps, dz, dy, dx);
        const int sz = z + dz, sy = y + dy, sx = x + dx;
        if (sz >= 0 && sz < a.d && sy >= 0 && sy < a.h && sx >= 0 && sx < a.w)
          val = gather8(a.s1, a.s2, grp, n, sz, sy, sx, a.d, a.h, a.w);
      }
      *reinterpret_cast<uint4*>(As + j16 * SBO + row_off) = val;
    }
#pragma unroll
    for (int j = 0; j < (COUT / 8 + 1) / 2; ++j) {
      const int nch = (tid >> 6) + 2 * j;
      if (nch < COUT / 8) {
        uint4 val = make_uint4(0, 0, 0, 0);
        if (valid) {
          val = ldg16(a.g + (size_t)v * COUT + nch * 8);
          if (a.gate) val = gate8(val, ldg16(a.gate + (size_t)v * COUT + nch * 8));
        }
        *reinterpret_cast<uint4*>(Bs + nch * SBO + row_off) = val;
      }
    }
    umma::fence_async_smem();
    ok = __syncthreads_and(ok);
    if (!ok) break;
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t a0 = umma::smem_addr(As), b0 = umma::smem_addr(Bs);
#pragma unroll
      for (int ks = 0; ks < kWgK / 16; ++ks)
        umma::mma(tmem, umma::desc(a0 + ks * 256, 128, SBO), umma::desc(b0 + ks * 256, 128, SBO), IDESC,
                  (st > 0 || ks > 0) ? 1u : 0u);
      umma::commit(&freeb[s]);
    }
  }
  if (tid == 0) umma::commit(done);
  const bool fin = umma::mbar_wait(done, 0);
  umma::fence_after_sync();
  if (__syncthreads_and(ok && fin)) {
    if (nst > 0) {
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
      const int mc = blockIdx.x * 16 + (tid >> 3);
      const bool mine = mc < mchunks;
      const int tap = mine ? mc / (CIN / 8) : 0;
      const int ci = mine ? (mc % (CIN / 8)) * 8 + (tid & 7) : 0;
#pragma unroll
      for (int c0 = 0; c0 < COUT; c0 += 16) {
        float f[16];
        umma::tmem_ld16(trow + c0, f);
        if (mine)
#pragma unroll
          for (int i = 0; i < 16; ++i) atomicAdd(&a.dw[((size_t)tap * COUT + c0 + i) * CIN + ci], f[i]);
      }
    }
  } else if (tid == 0) {
    atomicExch(a.err, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, TCOLS);
}

// ------------------------------------------------------------ other kernels
// db[c] += sum_v (g * gate)[v][c], C channels.
template <int C>
__global__ void k_bias_grad(const bf16* __restrict__ g, const bf16* __restrict__ gate, int V, float* db) {
  constexpr int G = C / 8;
  __shared__ float red[256][8];
  const int cg = threadIdx.x % G;
  const int lanes = 256 / G;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int v = blockIdx.x * lanes + threadIdx.x / G; v < V; v += gridDim.x * lanes) {
    uint4 q = ldg16(g + (size_t)v * C + cg * 8);
    if (gate) q = gate8(q, ldg16(gate + (size_t)v * C + cg * 8));
    const bf16* b = reinterpret_cast<const bf16*>(&q);
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] += __bfloat162float(b[i]);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) red[threadIdx.x][i] = acc[i];
  __syncthreads();
  if (threadIdx.x < G) {
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = threadIdx.x; t < lanes * G; t += G)
#pragma unroll
      for (int i = 0; i < 8; ++i) s[i] += red[t][i];
#pragma unroll
    for (int i = 0; i < 8; ++i) atomicAdd(&db[threadIdx.x * 8 + i], s[i]);
  }
}

// coarse[p] = scale * sum of the 8 children of p (fine grid d x h x w), C channels.
__global__ void k_pool(const bf16* __restrict__ fine, bf16* __restrict__ coarse, int n, int d, int h, int w, int C,
                       float scale) {
  const int G = C / 8;
  const int dc = d >> 1, hc = h >> 1, wc = w >> 1;
  const long total = (long)n * dc * hc * wc * G;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int cg = (int)(i % G);
    long p = i / G;
    const int x = (int)(p % wc);
    p /= wc;
    const int y = (int)(p % hc);
    p /= hc;
    const int z = (int)(p % dc);
    const int nn = (int)(p / dc);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < 8; ++c) {
      const size_t f = (((size_t)nn * d + 2 * z + (c >> 2)) * h + 2 * y + ((c >> 1) & 1)) * w + 2 * x + (c & 1);
      uint4 q = ldg16(fine + f * C + cg * 8);
      const bf16* b = reinterpret_cast<const bf16*>(&q);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] += __bfloat162float(b[k]);
    }
    uint4 out;
    uint32_t* o = reinterpret_cast<uint32_t*>(&out);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      __nv_bfloat162 b2 = __floats2bfloat162_rn(acc[2 * k] * scale, acc[2 * k + 1] * scale);
      o[k] = *reinterpret_cast<uint32_t*>(&b2);
    }
    const size_t cidx = (((size_t)nn * dc + z) * hc + y) * wc + x;
    *reinterpret_cast<uint4*>(coarse + cidx * C + cg * 8) = out;
  }
}

// fine[v] = (accumulate ? fine[v] : 0) + scale * coarse[parent(v)], C channels.
__global__ void k_unpool(const bf16* __restrict__ coarse, bf16* fine, int n, int d, int h, int w, int C, float scale,
                         int accumulate) {
  const int G = C / 8;
  const long total = (long)n * d * h * w * G;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int cg = (int)(i % G);
    long p = i / G;
    const int x = (int)(p % w);
    p /= w;
    const int y = (int)(p % h);
    p /= h;
    const int z = (int)(p % d);
    const int nn = (int)(p / d);
    const size_t cidx = (((size_t)nn * (d >> 1) + (z >> 1)) * (h >> 1) + (y >> 1)) * (w >> 1) + (x >> 1);
    uint4 q = ldg16(coarse + cidx * C + cg * 8);
    const bf16* b = reinterpret_cast<const bf16*>(&q);
    bf16* dst = fine + (((size_t)nn * d + z) * h + y) * w * C + (size_t)x * C + cg * 8;
    uint4 old = accumulate ? *reinterpret_cast<const uint4*>(dst) : make_uint4(0, 0, 0, 0);
    const bf16* ob = reinterpret_cast<const bf16*>(&old);
    uint4 out;
    uint32_t* o = reinterpret_cast<uint32_t*>(&out);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float f0 = __bfloat162float(ob[2 * k]) + scale * __bfloat162float(b[2 * k]);
      float f1 = __bfloat162float(ob[2 * k + 1]) + scale * __bfloat162float(b[2 * k + 1]);
      __nv_bfloat162 b2 = __floats2bfloat162_rn(f0, f1);
      o[k] = *reinterpret_cast<uint32_t*>(&b2);
    }
    *reinterpret_cast<uint4*>(dst) = out;
  }
}

// sums[2n] += sum over fluid voxels of r^2, sums[2n+1] += their count (sample n = blockIdx.y).
__global__ void k_rms(const float* __restrict__ r, const int8_t* __restrict__ m, int V1, double* sums) {
  const size_t base = (size_t)blockIdx.y * V1;
  double s = 0, c = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V1; i += gridDim.x * blockDim.x)
    if (m[base + i] == 1) {
      const double q = r[base + i];
      s += q * q;
      c += 1;
    }
  s = bsum(s);
  c = bsum(c);
  if (threadIdx.x == 0) {
    atomicAdd(&sums[2 * blockIdx.y], s);
    atomicAdd(&sums[2 * blockIdx.y + 1], c);
  }
}

__device__ __forceinline__ double sample_scale(const double* sums, int n) {
  const double c = sums[2 * n + 1];
  const double s = c > 0 ? sqrt(sums[2 * n] / c) : 0.0;
  return s > 0 ? s : 1.0;
}

// Network input: channel 0 = r / rms(r), channel 1 = mask (1 fluid, 0 air, -1 solid), 2..15 = 0.
__global__ void k_prep(const float* __restrict__ r, const int8_t* __restrict__ m, const double* sums, int V1,
                       bf16* in0) {
  const size_t base = (size_t)blockIdx.y * V1;
  const float inv = (float)(1.0 / sample_scale(sums, blockIdx.y));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V1; i += gridDim.x * blockDim.x) {
    const int8_t mk = m[base + i];
    const float rv = mk == 1 ? r[base + i] * inv : 0.0f;
    uint4 out = make_uint4(0, 0, 0, 0);
    __nv_bfloat162 b2 = __floats2bfloat162_rn(rv, (float)mk);
    out.x = *reinterpret_cast<uint32_t*>(&b2);
    uint4* dst = reinterpret_cast<uint4*>(in0 + (base + i) * 16);
    dst[0] = out;
    dst[1] = make_uint4(0, 0, 0, 0);
  }
}

// Mean squared error over the fluid voxels of the batch between the network
// output and e / (rms(r) * tscale); writes the output gradient (channel 0).
__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ e, const int8_t* __restrict__ m,
                       const double* sums, int nsamples, int V1, float tscale, bf16* gout, double* loss) {
  double total = 0;
  for (int k = 0; k < nsamples; ++k) total += sums[2 * k + 1];
  const double inv_count = total > 0 ? 1.0 / total : 0.0;
  const size_t base = (size_t)blockIdx.y * V1;
  const double tinv = 1.0 / (sample_scale(sums, blockIdx.y) * tscale);
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V1; i += gridDim.x * blockDim.x) {
    float gv = 0.0f;
    if (m[base + i] == 1) {
      const double diff = (double)out[base + i] - (double)e[base + i] * tinv;
      acc += diff * diff;
      gv = (float)(2.0 * diff * inv_count);
    }
    uint4 q = make_uint4(0, 0, 0, 0);
    __nv_bfloat162 b2 = __floats2bfloat162_rn(gv, 0.0f);
    q.x = *reinterpret_cast<uint32_t*>(&b2);
    uint4* dst = reinterpret_cast<uint4*>(gout + (base + i) * 16);
    dst[0] = q;
    dst[1] = make_uint4(0, 0, 0, 0);
  }
  acc = bsum(acc);
  if (threadIdx.x == 0) atomicAdd(loss, acc * inv_count);
}

// Energy-norm loss, first pass: d = out - e / (rms(r) tscale) on fluid voxels, 0 elsewhere.
__global__ void k_loss_diff(const float* __restrict__ out, const float* __restrict__ e, const int8_t* __restrict__ m,
                            const double* sums, int V1, float tscale, float* dbuf) {
  const size_t base = (size_t)blockIdx.y * V1;
  const double tinv = 1.0 / (sample_scale(sums, blockIdx.y) * tscale);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V1; i += gridDim.x * blockDim.x)
    dbuf[base + i] = m[base + i] == 1 ? (float)((double)out[base + i] - (double)e[base + i] * tinv) : 0.0f;
}

// Second pass: loss = sum over fluid voxels of d (M d) / count with M the
// unit-spacing operator of the mask (the one the training pairs solve), and
// the output gradient 2 (M d) / count (M is symmetric).
__global__ void k_loss_energy(const float* __restrict__ dbuf, const int8_t* __restrict__ m, const double* sums,
                              int nsamples, int d, int h, int w, bf16* gout, double* loss) {
  double total = 0;
  for (int k = 0; k < nsamples; ++k) total += sums[2 * k + 1];
  const double inv_count = total > 0 ? 1.0 / total : 0.0;
  const int V1 = d * h * w;
  const size_t base = (size_t)blockIdx.y * V1;
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V1; i += gridDim.x * blockDim.x) {
    float gv = 0.0f;
    if (m[base + i] == 1) {
      const int x = i % w, y = (i / w) % h, z = i / (w * h);
      const int c[3] = {x, y, z}, n[3] = {w, h, d}, stride[3] = {1, w, w * h};
      const double dc = dbuf[base + i];
      double q = 0;
      for (int a = 0; a < 3; ++a)
        for (int sgn = -1; sgn <= 1; sgn += 2) {
          const int cc = c[a] + sgn;
          if (cc < 0 || cc >= n[a]) continue;
          const size_t j = base + i + sgn * stride[a];
          if (m[j] == -1) continue;
          q += dc - (m[j] == 1 ? (double)dbuf[j] : 0.0);
        }
      acc += dc * q;
      gv = (float)(2.0 * q * inv_count);
    }
    uint4 qv = make_uint4(0, 0, 0, 0);
    __nv_bfloat162 b2 = __floats2bfloat162_rn(gv, 0.0f);
    qv.x = *reinterpret_cast<uint32_t*>(&b2);
    uint4* dst = reinterpret_cast<uint4*>(gout + (base + i) * 16);
    dst[0] = qv;
    dst[1] = make_uint4(0, 0, 0, 0);
  }
  acc = bsum(acc);
  if (threadIdx.x == 0) atomicAdd(loss, acc * inv_count);
}

// Correction in the units of r: z = out * rms(r) * tscale on fluid voxels, 0 elsewhere.
__global__ void k_out_scale(const float* __restrict__ out, const int8_t* __restrict__ m, const double* sums, int V1,
                            float tscale, float* z) {
  const size_t base = (size_t)blockIdx.y * V1;
  const float sc = (float)(sample_scale(sums, blockIdx.y) * tscale);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V1; i += gridDim.x * blockDim.x)
    z[base + i] = m[base + i] == 1 ? out[base + i] * sc : 0.0f;
}

__global__ void k_adam(float* p, const float* __restrict__ g, float* mo, float* ve, bf16* wb, long n, float lr,
                       float b1, float b2, float eps, float bc1, float bc2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    if (!isfinite(gi)) continue;  // a degenerate batch leaves the parameter as it is
    const float m1 = b1 * mo[i] + (1.0f - b1) * gi;
    const float v1 = b2 * ve[i] + (1.0f - b2) * gi * gi;
    mo[i] = m1;
    ve[i] = v1;
    const float pi = p[i] - lr * (m1 / bc1) / (sqrtf(v1 / bc2) + eps);
    p[i] = pi;
    wb[i] = __float2bfloat16_rn(pi);
  }
}

__global__ void k_cast(const float* __restrict__ p, bf16* wb, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    wb[i] = __float2bfloat16_rn(p[i]);
}

// --------------------------------------------------- training-pair generator
// Random fluid masks on an s^3 grid: fluid where z < pool_frac * s or inside one
// of the spheres (host-drawn centres and radii), air elsewhere; the grid's
// outside is solid.
__global__ void k_mask_gen(int8_t* m, const float* spheres, int nspheres, int s, float pool) {
  const size_t V1 = (size_t)s * s * s;
  const float* sp = spheres + (size_t)blockIdx.y * nspheres * 4;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % s), y = (int)((i / s) % s), z = (int)(i / ((size_t)s * s));
    bool f = z < pool;
    for (int k = 0; k < nspheres && !f; ++k) {
      const float dx = x - sp[4 * k], dy = y - sp[4 * k + 1], dz = z - sp[4 * k + 2];
      f = dx * dx + dy * dy + dz * dz <= sp[4 * k + 3] * sp[4 * k + 3];
    }
    m[blockIdx.y * V1 + i] = f ? 1 : 0;
  }
}

__device__ __forceinline__ double face_speed(uint64_t seed, uint64_t sample, size_t cell, int axis) {
  uint64_t k = seed ^ (sample * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)cell * 3 + axis) * 0xD1B54A32D192ED03ull;
  k ^= k >> 30;
  k *= 0xBF58476D1CE4E5B9ull;
  k ^= k >> 27;
  k *= 0x94D049BB133111EBull;
  k ^= k >> 31;
  return (double)(k >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Right-hand side of M x = rhs (M = -A, unit spacing): minus the divergence of
// random face speeds in [-1, 1]; faces on the grid's outside are zero (Neumann).
__global__ void k_rhs_gen(const int8_t* m, double* rhs, int s, uint64_t seed, uint64_t sample0) {
  const size_t V1 = (size_t)s * s * s;
  const size_t base = (size_t)blockIdx.y * V1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x) {
    const int c[3] = {(int)(i % s), (int)((i / s) % s), (int)(i / ((size_t)s * s))};
    double div = 0;
    if (m[base + i] == 1) {
      const size_t stride[3] = {1, (size_t)s, (size_t)s * s};
      for (int a = 0; a < 3; ++a) {
        const double lo = c[a] > 0 ? face_speed(seed, sample0 + blockIdx.y, i, a) : 0.0;
        const double hi = c[a] + 1 < s ? face_speed(seed, sample0 + blockIdx.y, i + stride[a], a) : 0.0;
        div += hi - lo;
      }
    }
    rhs[base + i] = -div;
  }
}

// q = M p (unit spacing), pq[n] += p.q over the sample's fluid voxels.
__global__ void k_cg_apply(const int8_t* __restrict__ m, const double* __restrict__ p, double* q, int s,
                           double* pq) {
  const size_t V1 = (size_t)s * s * s;
  const size_t base = (size_t)blockIdx.y * V1;
  double acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x) {
    double out = 0;
    if (m[base + i] == 1) {
      const int c[3] = {(int)(i % s), (int)((i / s) % s), (int)(i / ((size_t)s * s))};
      const size_t stride[3] = {1, (size_t)s, (size_t)s * s};
      const double pc = p[base + i];
      for (int a = 0; a < 3; ++a) {
        if (c[a] > 0) {
          const size_t j = base + i - stride[a];
          out += pc - (m[j] == 1 ? p[j] : 0.0);
        }
        if (c[a] + 1 < s) {
          const size_t j = base + i + stride[a];
          out += pc - (m[j] == 1 ? p[j] : 0.0);
        }
      }
      acc += pc * out;
    }
    q[base + i] = out;
  }
  acc = bsum(acc);
  if (threadIdx.x == 0) atomicAdd(&pq[blockIdx.y], acc);
}

// x += alpha p, r -= alpha q, rr[n] += r.r (alpha = rr_old / pq per sample).
__global__ void k_cg_xr(double* x, double* r, const double* __restrict__ p, const double* __restrict__ q,
                        const double* rr_old, const double* pq, double* rr_new, size_t V1) {
  const size_t base = (size_t)blockIdx.y * V1;
  const double alpha = pq[blockIdx.y] > 0 ? rr_old[blockIdx.y] / pq[blockIdx.y] : 0.0;
  double acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x) {
    x[base + i] += alpha * p[base + i];
    const double rv = r[base + i] - alpha * q[base + i];
    r[base + i] = rv;
    acc += rv * rv;
  }
  acc = bsum(acc);
  if (threadIdx.x == 0) atomicAdd(&rr_new[blockIdx.y], acc);
}

// p = r + (rr_new / rr_old) p
__global__ void k_cg_p(double* p, const double* __restrict__ r, const double* rr_old, const double* rr_new,
                       size_t V1) {
  const size_t base = (size_t)blockIdx.y * V1;
  const double beta = rr_old[blockIdx.y] > 0 ? rr_new[blockIdx.y] / rr_old[blockIdx.y] : 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x)
    p[base + i] = r[base + i] + beta * p[base + i];
}

__global__ void k_dot_self(const double* __restrict__ r, size_t V1, double* out) {
  const size_t base = (size_t)blockIdx.y * V1;
  double acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x)
    acc += r[base + i] * r[base + i];
  acc = bsum(acc);
  if (threadIdx.x == 0) atomicAdd(&out[blockIdx.y], acc);
}

__global__ void k_to_f32(const double* __restrict__ a, float* b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// e = x_final - x_snapshot (FP32)
__global__ void k_err(const double* __restrict__ xf, const double* __restrict__ xs, float* e, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    e[i] = (float)(xf[i] - xs[i]);
}

// sums[0] += sum over fluid voxels of (e / rms(r))^2, sums[1] += count, over samples blockIdx.y.
__global__ void k_target_stats(const float* __restrict__ r, const float* __restrict__ e, const int8_t* __restrict__ m,
                               const double* rsums, size_t V1, double* out) {
  const size_t base = (size_t)blockIdx.y * V1;
  const double inv = 1.0 / sample_scale(rsums, blockIdx.y);
  double s = 0, c = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x)
    if (m[base + i] == 1) {
      const double q = e[base + i] * inv;
      s += q * q;
      c += 1;
    }
  s = bsum(s);
  c = bsum(c);
  if (threadIdx.x == 0) {
    atomicAdd(&out[0], s);
    atomicAdd(&out[1], c);
  }
}

// Copies the samples idx[k] = hash(seed, step, k) mod count into the batch buffers.
__global__ void k_gather_batch(const float* __restrict__ dr, const float* __restrict__ de,
                               const int8_t* __restrict__ dm, int count, size_t V1, uint64_t seed, uint64_t step,
                               float* r, float* e, int8_t* m) {
  uint64_t k = seed * 0x9E3779B97F4A7C15ull + step * 0xBF58476D1CE4E5B9ull + blockIdx.y * 0x94D049BB133111EBull;
  k ^= k >> 31;
  k *= 0xD6E8FEB86659FD93ull;
  k ^= k >> 32;
  const size_t src = (size_t)(k % (uint64_t)count) * V1, dst = (size_t)blockIdx.y * V1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < V1; i += (size_t)gridDim.x * blockDim.x) {
    r[dst + i] = dr[src + i];
    e[dst + i] = de[src + i];
    m[dst + i] = dm[src + i];
  }
}

}  // namespace unet
}  // namespace mac

// ===================================================================== host
namespace mac {
namespace unet {

static int cuda_ok(cudaError_t e) { return e == cudaSuccess ? MAC_OK : (e == cudaErrorMemoryAllocation ? MAC_ERR_OUT_OF_MEMORY : MAC_ERR_CUDA); }

static int grid_1d(size_t n, int threads = 256) {
  size_t g = (n + threads - 1) / threads;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

template <int KC, int NC, int MODE>
static void conv_t(const ConvArgs& a, cudaStream_t st) {
  const int smem = conv_smem<KC, NC>();
  cudaFuncSetAttribute(k_conv<KC, NC, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const long V = (long)a.n * a.d * a.h * a.w;
  k_conv<KC, NC, MODE><<<(unsigned)((V + 127) / 128), 128, smem, st>>>(a);
}

template <int KC, int NC>
static void conv_tile_t(const ConvArgs& a, cudaStream_t st) {
  const int smem = tile_smem<KC, NC>();
  cudaFuncSetAttribute(k_conv_tile<KC, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const long tiles = (long)a.n * a.d * ((a.h + 15) / 16) * ((a.w + 7) / 8);
  k_conv_tile<KC, NC><<<(unsigned)tiles, 128, smem, st>>>(a);
}

// Forward 3x3x3 convolutions through the staged-tile kernel.
static int conv_tile(int kc, int nc, const ConvArgs& a, cudaStream_t st) {
  if (kc == 16 && nc == 16) conv_tile_t<16, 16>(a, st);
  else if (kc == 16 && nc == 32) conv_tile_t<16, 32>(a, st);
  else if (kc == 32 && nc == 32) conv_tile_t<32, 32>(a, st);
  else if (kc == 32 && nc == 64) conv_tile_t<32, 64>(a, st);
  else if (kc == 64 && nc == 64) conv_tile_t<64, 64>(a, st);
  else if (kc == 64 && nc == 32) conv_tile_t<64, 32>(a, st);
  else if (kc == 32 && nc == 16) conv_tile_t<32, 16>(a, st);
  else return MAC_ERR_INVALID;
  return MAC_OK;
}

template <int MODE>
static int conv_mode(int kc, int nc, const ConvArgs& a, cudaStream_t st) {
  if (kc == 16 && nc == 16) conv_t<16, 16, MODE>(a, st);
  else if (kc == 16 && nc == 32) conv_t<16, 32, MODE>(a, st);
  else if (kc == 32 && nc == 32) conv_t<32, 32, MODE>(a, st);
  else if (kc == 32 && nc == 64) conv_t<32, 64, MODE>(a, st);
  else if (kc == 64 && nc == 64) conv_t<64, 64, MODE>(a, st);
  else if (kc == 64 && nc == 32) conv_t<64, 32, MODE>(a, st);
  else if (kc == 32 && nc == 16) conv_t<32, 16, MODE>(a, st);
  else return MAC_ERR_INVALID;
  return MAC_OK;
}

template <int CIN, int COUT>
static void wgrad_t(const WgradArgs& a, cudaStream_t st) {
  const int smem = wgrad_smem<CIN, COUT>();
  cudaFuncSetAttribute(k_wgrad<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const long V = (long)a.n * a.d * a.h * a.w;
  const int mtiles = (a.taps * (CIN / 8) + 15) / 16;
  const int ksplit = (int)((V + a.vox_per_cta - 1) / a.vox_per_cta);
  k_wgrad<CIN, COUT><<<dim3(mtiles, ksplit), 128, smem, st>>>(a);
}

static int wgrad(int cin, int cout, WgradArgs a, cudaStream_t st) {
  const long V = (long)a.n * a.d * a.h * a.w;
  const int mtiles = (a.taps * (cin / 8) + 15) / 16;
  long ksplit = (296 + mtiles - 1) / mtiles;
  const long maxsplit = (V + 255) / 256;
  if (ksplit > maxsplit) ksplit = maxsplit;
  if (ksplit < 1) ksplit = 1;
  long per = (V + ksplit - 1) / ksplit;
  a.vox_per_cta = (int)((per + kWgK - 1) / kWgK * kWgK);
  if (cin == 16 && cout == 16) wgrad_t<16, 16>(a, st);
  else if (cin == 16 && cout == 32) wgrad_t<16, 32>(a, st);
  else if (cin == 32 && cout == 32) wgrad_t<32, 32>(a, st);
  else if (cin == 32 && cout == 64) wgrad_t<32, 64>(a, st);
  else if (cin == 64 && cout == 64) wgrad_t<64, 64>(a, st);
  else if (cin == 64 && cout == 32) wgrad_t<64, 32>(a, st);
  else if (cin == 32 && cout == 16) wgrad_t<32, 16>(a, st);
  else return MAC_ERR_INVALID;
  return MAC_OK;
}

static void bias_grad(int c, const bf16* g, const bf16* gate, long V, float* db, cudaStream_t st) {
  const int blocks = (int)std::min<long>(296, (V * (c / 8) + 255) / 256);
  if (c == 16) k_bias_grad<16><<<blocks, 256, 0, st>>>(g, gate, (int)V, db);
  else if (c == 32) k_bias_grad<32><<<blocks, 256, 0, st>>>(g, gate, (int)V, db);
  else k_bias_grad<64><<<blocks, 256, 0, st>>>(g, gate, (int)V, db);
}

struct Net {
  int device = 0;
  size_t woff[kNumLayers] = {}, boff[kNumLayers] = {};
  size_t np = 0;
  float *p = nullptr, *g = nullptr, *mo = nullptr, *ve = nullptr;
  bf16* wb = nullptr;
  long adam_t = 0;
  float tscale = 1.0f;
  int loss_kind = 0;  // 0: mean squared error, 1: energy norm of the error
  int n = 0, d = 0, h = 0, w = 0;
  size_t cap = 0;  // level-0 voxels the shape buffers hold
  bf16* act[kNumAct] = {};
  bf16* grad[kNumAct] = {};
  float *out = nullptr, *r = nullptr, *e = nullptr, *dbuf = nullptr;
  int8_t* m = nullptr;
  double *sums = nullptr, *loss = nullptr;
  int* err = nullptr;
  int ds_size = 0, ds_count = 0;
  float *ds_r = nullptr, *ds_e = nullptr;
  int8_t* ds_m = nullptr;
  double* loss_hist = nullptr;
  int loss_cap = 0;
  long launches = 0;
  int staged_conv = 1;  // forward 3x3x3 convolutions through k_conv_tile (0: k_conv)
};

static size_t level_vox(const Net& t, int l) {
  return (size_t)t.n * (t.d >> l) * (t.h >> l) * (t.w >> l);
}

static void free_shape(Net& t) {
  for (int i = 0; i < kNumAct; ++i) {
    cudaFree(t.act[i]);
    cudaFree(t.grad[i]);
    t.act[i] = t.grad[i] = nullptr;
  }
  cudaFree(t.out);
  cudaFree(t.r);
  cudaFree(t.e);
  cudaFree(t.m);
  cudaFree(t.dbuf);
  t.out = t.r = t.e = t.dbuf = nullptr;
  t.m = nullptr;
  t.cap = 0;
}

// Sizes the activation buffers for n samples on a d x h x w grid (each a multiple of 4).
static int ensure_shape(Net& t, int n, int d, int h, int w) {
  if (n < 1 || d < 4 || h < 4 || w < 4 || d % 4 || h % 4 || w % 4) return MAC_ERR_INVALID;
  const size_t v0 = (size_t)n * d * h * w;
  if (v0 > (size_t)INT32_MAX / 64) return MAC_ERR_CAPACITY;
  if (v0 > t.cap) {
    free_shape(t);
    t.n = n;
    t.d = d;
    t.h = h;
    t.w = w;
    int rc = MAC_OK;
    for (int i = 0; i < kNumAct && !rc; ++i) {
      const size_t bytes = level_vox(t, kActLvl[i]) * kActCh[i] * sizeof(bf16);
      rc = cuda_ok(cudaMalloc((void**)&t.act[i], bytes));
      if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.grad[i], bytes));
    }
    if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.out, v0 * 4));
    if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.r, v0 * 4));
    if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.e, v0 * 4));
    if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.m, v0));
    if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.dbuf, v0 * 4));
    if (rc) {
      free_shape(t);
      return rc;
    }
    t.cap = v0;
  }
  t.n = n;
  t.d = d;
  t.h = h;
  t.w = w;
  return MAC_OK;
}

// Convolution arguments of layer l on the grid of level lvl.
static ConvArgs conv_args(Net& t, int l, int lvl) {
  ConvArgs a;
  std::memset(&a, 0, sizeof(a));
  a.wt = t.wb + t.woff[l];
  a.taps = kLayers[l].taps;
  a.n = t.n;
  a.d = t.d >> lvl;
  a.h = t.h >> lvl;
  a.w = t.w >> lvl;
  a.err = t.err;
  return a;
}

static Src src(const bf16* p, int c, int shift = 0) { return Src{p, c, shift}; }
static Src none() { return Src{nullptr, 0, 0}; }

// Forward convolution of layer l: out = act(conv(concat(s1, s2)) + bias).
static int fwd(Net& t, int l, int lvl, Src s1, Src s2, bf16* dst, float* f32, cudaStream_t st) {
  ConvArgs a = conv_args(t, l, lvl);
  a.s1 = s1;
  a.s2 = s2;
  a.bias = t.p + t.boff[l];
  a.d1 = dst;
  a.c1 = kLayers[l].cout;
  a.f32 = f32;
  a.relu = kLayers[l].relu;
  ++t.launches;
  if (t.staged_conv && a.taps == 27) return conv_tile(kLayers[l].cin, kLayers[l].cout, a, st);
  return conv_mode<0>(kLayers[l].cin, kLayers[l].cout, a, st);
}

// Input gradient of layer l from the gradient g at its output (gated by the
// layer's ReLU output y when it has one); channels [0, c1) to d1, the rest to d2.
static int bwd_in(Net& t, int l, int lvl, const bf16* g, const bf16* y, bf16* d1, int c1, bf16* d2,
                  cudaStream_t st) {
  ConvArgs a = conv_args(t, l, lvl);
  a.s1 = src(g, kLayers[l].cout);
  a.s2 = none();
  a.gate = kLayers[l].relu ? y : nullptr;
  a.d1 = d1;
  a.c1 = c1;
  a.d2 = d2;
  ++t.launches;
  return conv_mode<1>(kLayers[l].cout, kLayers[l].cin, a, st);
}

// Weight and bias gradients of layer l (input concat(s1, s2), output gradient g, output y).
static int bwd_w(Net& t, int l, int lvl, Src s1, Src s2, const bf16* g, const bf16* y, cudaStream_t st) {
  WgradArgs a;
  std::memset(&a, 0, sizeof(a));
  a.s1 = s1;
  a.s2 = s2;
  a.g = g;
  a.gate = kLayers[l].relu ? y : nullptr;
  a.dw = t.g + t.woff[l];
  a.taps = kLayers[l].taps;
  a.n = t.n;
  a.d = t.d >> lvl;
  a.h = t.h >> lvl;
  a.w = t.w >> lvl;
  a.err = t.err;
  t.launches += 2;
  int rc = wgrad(kLayers[l].cin, kLayers[l].cout, a, st);
  bias_grad(kLayers[l].cout, g, a.gate, (long)a.n * a.d * a.h * a.w, t.g + t.boff[l], st);
  return rc;
}

static void pool(Net& t, int lvl, const bf16* fine, bf16* coarse, int c, float scale, cudaStream_t st) {
  const size_t n = level_vox(t, lvl + 1) * (c / 8);
  k_pool<<<grid_1d(n), 256, 0, st>>>(fine, coarse, t.n, t.d >> lvl, t.h >> lvl, t.w >> lvl, c, scale);
  ++t.launches;
}

static void unpool(Net& t, int lvl, const bf16* coarse, bf16* fine, int c, float scale, int acc, cudaStream_t st) {
  const size_t n = level_vox(t, lvl) * (c / 8);
  k_unpool<<<grid_1d(n), 256, 0, st>>>(coarse, fine, t.n, t.d >> lvl, t.h >> lvl, t.w >> lvl, c, scale, acc);
  ++t.launches;
}

static int forward(Net& t, cudaStream_t st) {
  bf16** A = t.act;
  int rc = 0;
  rc |= fwd(t, 0, 0, src(A[IN0], 16), none(), A[A1], nullptr, st);
  rc |= fwd(t, 1, 0, src(A[A1], 16), none(), A[S1], nullptr, st);
  pool(t, 0, A[S1], A[P1], 16, 0.125f, st);
  rc |= fwd(t, 2, 1, src(A[P1], 16), none(), A[A2], nullptr, st);
  rc |= fwd(t, 3, 1, src(A[A2], 32), none(), A[S2], nullptr, st);
  pool(t, 1, A[S2], A[P2], 32, 0.125f, st);
  rc |= fwd(t, 4, 2, src(A[P2], 32), none(), A[A3], nullptr, st);
  rc |= fwd(t, 5, 2, src(A[A3], 64), none(), A[B3], nullptr, st);
  rc |= fwd(t, 6, 2, src(A[B3], 64), none(), A[U2], nullptr, st);
  rc |= fwd(t, 7, 1, src(A[S2], 32), src(A[U2], 32, 1), A[C2], nullptr, st);
  rc |= fwd(t, 8, 1, src(A[C2], 32), none(), A[D2], nullptr, st);
  rc |= fwd(t, 9, 1, src(A[D2], 32), none(), A[U1], nullptr, st);
  rc |= fwd(t, 10, 0, src(A[S1], 16), src(A[U1], 16, 1), A[C1], nullptr, st);
  rc |= fwd(t, 11, 0, src(A[C1], 16), none(), A[D1], nullptr, st);
  rc |= fwd(t, 12, 0, src(A[D1], 16), none(), nullptr, t.out, st);
  return rc ? MAC_ERR_INVALID : MAC_OK;
}

// Gradients of every parameter into t.g (zeroed first) from the output
// gradient in grad[GOUT].
static int backward(Net& t, cudaStream_t st) {
  bf16** A = t.act;
  bf16** G = t.grad;
  int rc = cuda_ok(cudaMemsetAsync(t.g, 0, t.np * sizeof(float), st));
  rc |= bwd_w(t, 12, 0, src(A[D1], 16), none(), G[GOUT], nullptr, st);
  rc |= bwd_in(t, 12, 0, G[GOUT], nullptr, G[D1], 16, nullptr, st);
  rc |= bwd_w(t, 11, 0, src(A[C1], 16), none(), G[D1], A[D1], st);
  rc |= bwd_in(t, 11, 0, G[D1], A[D1], G[C1], 16, nullptr, st);
  rc |= bwd_w(t, 10, 0, src(A[S1], 16), src(A[U1], 16, 1), G[C1], A[C1], st);
  rc |= bwd_in(t, 10, 0, G[C1], A[C1], G[S1], 16, G[GUP1], st);
  pool(t, 0, G[GUP1], G[U1], 16, 1.0f, st);
  rc |= bwd_w(t, 9, 1, src(A[D2], 32), none(), G[U1], nullptr, st);
  rc |= bwd_in(t, 9, 1, G[U1], nullptr, G[D2], 32, nullptr, st);
  rc |= bwd_w(t, 8, 1, src(A[C2], 32), none(), G[D2], A[D2], st);
  rc |= bwd_in(t, 8, 1, G[D2], A[D2], G[C2], 32, nullptr, st);
  rc |= bwd_w(t, 7, 1, src(A[S2], 32), src(A[U2], 32, 1), G[C2], A[C2], st);
  rc |= bwd_in(t, 7, 1, G[C2], A[C2], G[S2], 32, G[GUP2], st);
  pool(t, 1, G[GUP2], G[U2], 32, 1.0f, st);
  rc |= bwd_w(t, 6, 2, src(A[B3], 64), none(), G[U2], nullptr, st);
  rc |= bwd_in(t, 6, 2, G[U2], nullptr, G[B3], 64, nullptr, st);
  rc |= bwd_w(t, 5, 2, src(A[A3], 64), none(), G[B3], A[B3], st);
  rc |= bwd_in(t, 5, 2, G[B3], A[B3], G[A3], 64, nullptr, st);
  rc |= bwd_w(t, 4, 2, src(A[P2], 32), none(), G[A3], A[A3], st);
  rc |= bwd_in(t, 4, 2, G[A3], A[A3], G[P2], 32, nullptr, st);
  unpool(t, 1, G[P2], G[S2], 32, 0.125f, 1, st);
  rc |= bwd_w(t, 3, 1, src(A[A2], 32), none(), G[S2], A[S2], st);
  rc |= bwd_in(t, 3, 1, G[S2], A[S2], G[A2], 32, nullptr, st);
  rc |= bwd_w(t, 2, 1, src(A[P1], 16), none(), G[A2], A[A2], st);
  rc |= bwd_in(t, 2, 1, G[A2], A[A2], G[P1], 16, nullptr, st);
  unpool(t, 0, G[P1], G[S1], 16, 0.125f, 1, st);
  rc |= bwd_w(t, 1, 0, src(A[A1], 16), none(), G[S1], A[S1], st);
  rc |= bwd_in(t, 1, 0, G[S1], A[S1], G[A1], 16, nullptr, st);
  rc |= bwd_w(t, 0, 0, src(A[IN0], 16), none(), G[A1], A[A1], st);
  return rc ? MAC_ERR_INVALID : MAC_OK;
}

// Network input from t.r / t.m (n samples on the current grid); per-sample rms in t.sums.
static void prep(Net& t, cudaStream_t st) {
  const int V1 = t.d * t.h * t.w;
  cudaMemsetAsync(t.sums, 0, 2 * sizeof(double) * t.n, st);
  const dim3 g((V1 + 255) / 256 < 148 ? (V1 + 255) / 256 : 148, t.n);
  k_rms<<<g, 256, 0, st>>>(t.r, t.m, V1, t.sums);
  k_prep<<<g, 256, 0, st>>>(t.r, t.m, t.sums, V1, t.act[IN0]);
  t.launches += 2;
}

static int check_err(Net& t, cudaStream_t st) {
  int h = 0;
  int rc = cuda_ok(cudaMemcpyAsync(&h, t.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (!rc) rc = cuda_ok(cudaStreamSynchronize(st));
  if (!rc) rc = cuda_ok(cudaGetLastError());
  if (!rc && h) {
    cudaMemsetAsync(t.err, 0, sizeof(int), st);
    rc = MAC_ERR_TIMEOUT;
  }
  return rc;
}

static void layer_offsets(Net& t) {
  size_t o = 0;
  for (int l = 0; l < kNumLayers; ++l) {
    t.woff[l] = o;
    o += (size_t)kLayers[l].taps * kLayers[l].cout * kLayers[l].cin;
    t.boff[l] = o;
    o += kLayers[l].cout;
    o = (o + 7) / 8 * 8;  // keeps every weight block 16-byte aligned in BF16
  }
  t.np = o;
}

static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double uniform(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

// He-uniform weights over the real (unpadded) channels, zero biases and padding.
static std::vector<float> init_params(const Net& t, uint64_t seed) {
  std::vector<float> p(t.np, 0.0f);
  uint64_t s = seed;
  for (int l = 0; l < kNumLayers; ++l) {
    const LayerDef& L = kLayers[l];
    const double fan_in = (double)L.taps * L.real_cin;
    const double b = std::sqrt((L.relu ? 6.0 : 3.0) / fan_in);
    for (int tp = 0; tp < L.taps; ++tp)
      for (int co = 0; co < L.real_cout; ++co)
        for (int ci = 0; ci < L.real_cin; ++ci)
          p[t.woff[l] + ((size_t)tp * L.cout + co) * L.cin + ci] = (float)((2.0 * uniform(s) - 1.0) * b);
  }
  return p;
}

static int set_params(Net& t, const float* host, cudaStream_t st) {
  int rc = cuda_ok(cudaMemcpyAsync(t.p, host, t.np * 4, cudaMemcpyHostToDevice, st));
  if (rc) return rc;
  k_cast<<<grid_1d(t.np), 256, 0, st>>>(t.p, t.wb, (long)t.np);
  cudaMemsetAsync(t.mo, 0, t.np * 4, st);
  cudaMemsetAsync(t.ve, 0, t.np * 4, st);
  t.adam_t = 0;
  return cuda_ok(cudaStreamSynchronize(st));
}

void destroy(Net* t);

static int create(int device, Net** out) {
  Net* t = new Net();
  t->device = device;
  layer_offsets(*t);
  int rc = cuda_ok(cudaSetDevice(device));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->p, t->np * 4));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->g, t->np * 4));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->mo, t->np * 4));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->ve, t->np * 4));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->wb, t->np * 2));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->sums, 2 * sizeof(double) * 65536));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->loss, sizeof(double)));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t->err, sizeof(int)));
  if (!rc) rc = cuda_ok(cudaMemset(t->err, 0, sizeof(int)));
  if (!rc) {
    std::vector<float> p = init_params(*t, 1);
    rc = set_params(*t, p.data(), 0);
  }
  if (rc) {
    destroy(t);
    return rc;
  }
  *out = t;
  return MAC_OK;
}

void destroy(Net* t) {
  if (!t) return;
  cudaSetDevice(t->device);
  free_shape(*t);
  cudaFree(t->p);
  cudaFree(t->g);
  cudaFree(t->mo);
  cudaFree(t->ve);
  cudaFree(t->wb);
  cudaFree(t->sums);
  cudaFree(t->loss);
  cudaFree(t->err);
  cudaFree(t->ds_r);
  cudaFree(t->ds_e);
  cudaFree(t->ds_m);
  cudaFree(t->loss_hist);
  delete t;
}

// Correction of the residuals in t.r (masks t.m) on the current grid into t.e:
// z = net(r / rms(r)) * rms(r) * tscale on fluid voxels. Unit cell spacing.
int apply(Net* t, cudaStream_t st) {
  prep(*t, st);
  int rc = forward(*t, st);
  const int V1 = t->d * t->h * t->w;
  const dim3 g((V1 + 255) / 256 < 148 ? (V1 + 255) / 256 : 148, t->n);
  k_out_scale<<<g, 256, 0, st>>>(t->out, t->m, t->sums, V1, t->tscale, t->e);
  ++t->launches;
  return rc;
}

// Loss of the batch in t.r / t.m / t.e into *loss_dst (device) and all parameter gradients.
static int loss_grad(Net& t, double* loss_dst, cudaStream_t st) {
  prep(t, st);
  int rc = forward(t, st);
  const int V1 = t.d * t.h * t.w;
  cudaMemsetAsync(loss_dst, 0, sizeof(double), st);
  const dim3 g((V1 + 255) / 256 < 148 ? (V1 + 255) / 256 : 148, t.n);
  if (t.loss_kind == 1) {
    k_loss_diff<<<g, 256, 0, st>>>(t.out, t.e, t.m, t.sums, V1, t.tscale, t.dbuf);
    k_loss_energy<<<g, 256, 0, st>>>(t.dbuf, t.m, t.sums, t.n, t.d, t.h, t.w, t.grad[GOUT], loss_dst);
    t.launches += 2;
  } else {
    k_loss<<<g, 256, 0, st>>>(t.out, t.e, t.m, t.sums, t.n, V1, t.tscale, t.grad[GOUT], loss_dst);
    ++t.launches;
  }
  if (!rc) rc = backward(t, st);
  return rc;
}

static void adam(Net& t, float lr, cudaStream_t st) {
  ++t.adam_t;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.0f - std::pow(b1, (float)t.adam_t), bc2 = 1.0f - std::pow(b2, (float)t.adam_t);
  k_adam<<<grid_1d(t.np), 256, 0, st>>>(t.p, t.g, t.mo, t.ve, t.wb, (long)t.np, lr, b1, b2, 1e-8f, bc1, bc2);
  ++t.launches;
}

// Training pairs: nmasks random masks on an s^3 grid, each solved by plain FP64
// CG from x = 0 for niter iterations; the residual r_k and the error
// x_final - x_k at iterations k = 1, 2, 4, ... (nsnap of them) are kept.
// Sample index = snapshot * nmasks + mask. stats: [0] largest final relative
// residual, [1] target scale.
// The first next masks come from ext (next x s^3 host bytes: 1 fluid, 0 air
// or missing, -1 solid), the rest are random pools with spheres.
static int make_dataset(Net& t, int nmasks, int s, int nsnap, int niter, uint64_t seed, double* stats,
                        cudaStream_t st, const int8_t* ext = nullptr, int next = 0) {
  if (nmasks < 1 || s < 8 || s % 4 || nsnap < 1 || nsnap > 16 || niter < (1 << (nsnap - 1))) return MAC_ERR_INVALID;
  const size_t V1 = (size_t)s * s * s;
  const size_t S = (size_t)nmasks * nsnap;
  cudaFree(t.ds_r);
  cudaFree(t.ds_e);
  cudaFree(t.ds_m);
  t.ds_r = t.ds_e = nullptr;
  t.ds_m = nullptr;
  t.ds_count = 0;
  int rc = cuda_ok(cudaMalloc((void**)&t.ds_r, S * V1 * 4));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.ds_e, S * V1 * 4));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&t.ds_m, S * V1));
  if (rc) return rc;
  const int MB = std::min(nmasks, 32);
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *xs = nullptr, *sc = nullptr;
  int8_t* m = nullptr;
  float* sph = nullptr;
  const int nsph = 12;
  rc = cuda_ok(cudaMalloc((void**)&x, MB * V1 * 8));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&r, MB * V1 * 8));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&p, MB * V1 * 8));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&q, MB * V1 * 8));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&xs, (size_t)nsnap * MB * V1 * 8));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&sc, 4 * MB * sizeof(double) + 64));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&m, MB * V1));
  if (!rc) rc = cuda_ok(cudaMalloc((void**)&sph, (size_t)MB * nsph * 4 * sizeof(float)));
  double worst = 0;
  uint64_t rs = seed;
  const dim3 g1((unsigned)std::min<size_t>((V1 + 255) / 256, 296), MB);
  for (int m0 = 0; m0 < nmasks && !rc; m0 += MB) {
    const int nb = std::min(MB, nmasks - m0);
    std::vector<float> hs((size_t)MB * nsph * 4);
    const double scale = s / 64.0;
    for (int b = 0; b < nb; ++b)
      for (int k = 0; k < nsph; ++k) {
        const double rad = (3.0 + 7.0 * uniform(rs)) * scale;
        float* o = &hs[((size_t)b * nsph + k) * 4];
        for (int a = 0; a < 3; ++a) o[a] = (float)(rad + (s - 2 * rad) * uniform(rs));
        o[3] = (float)rad;
      }
    cudaMemcpyAsync(sph, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, st);
    const dim3 g(g1.x, nb);
    double *rr = sc, *rrn = sc + MB, *pq = sc + 2 * MB, *rr0 = sc + 3 * MB;
    k_mask_gen<<<g, 256, 0, st>>>(m, sph, nsph, s, (float)(0.4 * s));
    for (int b = 0; b < nb; ++b)
      if (m0 + b < next) cudaMemcpyAsync(m + (size_t)b * V1, ext + (size_t)(m0 + b) * V1, V1, cudaMemcpyHostToDevice, st);
    k_rhs_gen<<<g, 256, 0, st>>>(m, r, s, seed, (uint64_t)m0);
    cudaMemsetAsync(x, 0, nb * V1 * 8, st);
    cudaMemcpyAsync(p, r, nb * V1 * 8, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(sc, 0, 4 * MB * sizeof(double), st);
    k_dot_self<<<g, 256, 0, st>>>(r, V1, rr);
    cudaMemcpyAsync(rr0, rr, MB * sizeof(double), cudaMemcpyDeviceToDevice, st);
    int snap = 0;
    for (int it = 1; it <= niter; ++it) {
      cudaMemsetAsync(pq, 0, MB * sizeof(double), st);
      cudaMemsetAsync(rrn, 0, MB * sizeof(double), st);
      k_cg_apply<<<g, 256, 0, st>>>(m, p, q, s, pq);
      k_cg_xr<<<g, 256, 0, st>>>(x, r, p, q, rr, pq, rrn, V1);
      k_cg_p<<<g, 256, 0, st>>>(p, r, rr, rrn, V1);
      std::swap(rr, rrn);
      if (snap < nsnap && it == (1 << snap)) {
        const size_t row = (size_t)snap * nmasks + m0;
        k_to_f32<<<grid_1d(nb * V1), 256, 0, st>>>(r, t.ds_r + row * V1, nb * V1);
        cudaMemcpyAsync(xs + (size_t)snap * MB * V1, x, nb * V1 * 8, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(t.ds_m + row * V1, m, nb * V1, cudaMemcpyDeviceToDevice, st);
        ++snap;
      }
    }
    for (int j = 0; j < nsnap; ++j) {
      const size_t row = (size_t)j * nmasks + m0;
      k_err<<<grid_1d(nb * V1), 256, 0, st>>>(x, xs + (size_t)j * MB * V1, t.ds_e + row * V1, nb * V1);
    }
    std::vector<double> h(2 * MB);
    cudaMemcpyAsync(h.data(), rr, MB * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h.data() + MB, rr0, MB * sizeof(double), cudaMemcpyDeviceToHost, st);
    rc = cuda_ok(cudaStreamSynchronize(st));
    for (int b = 0; b < nb && !rc; ++b)
      if (h[MB + b] > 0) worst = std::max(worst, std::sqrt(h[b] / h[MB + b]));
  }
  cudaFree(x);
  cudaFree(r);
  cudaFree(p);
  cudaFree(q);
  cudaFree(xs);
  cudaFree(m);
  cudaFree(sph);
  if (!rc) {
    // target scale: rms of e / rms(r) over the whole set
    double* rsum = nullptr;
    rc = cuda_ok(cudaMalloc((void**)&rsum, (2 * S + 2) * sizeof(double)));
    if (!rc) {
      cudaMemsetAsync(rsum, 0, (2 * S + 2) * sizeof(double), st);
      for (size_t s0 = 0; s0 < S; s0 += 65535) {
        const unsigned ny = (unsigned)std::min<size_t>(65535, S - s0);
        const dim3 g(g1.x, ny);
        k_rms<<<g, 256, 0, st>>>(t.ds_r + s0 * V1, t.ds_m + s0 * V1, (int)V1, rsum + 2 * s0);
        k_target_stats<<<g, 256, 0, st>>>(t.ds_r + s0 * V1, t.ds_e + s0 * V1, t.ds_m + s0 * V1, rsum + 2 * s0, V1,
                                          rsum + 2 * S);
      }
      double h2[2] = {0, 0};
      cudaMemcpyAsync(h2, rsum + 2 * S, 16, cudaMemcpyDeviceToHost, st);
      rc = cuda_ok(cudaStreamSynchronize(st));
      if (!rc && h2[1] > 0) t.tscale = (float)std::sqrt(h2[0] / h2[1]);
      cudaFree(rsum);
    }
  }
  cudaFree(sc);
  if (rc) return rc;
  t.ds_count = (int)S;
  t.ds_size = s;
  if (stats) {
    stats[0] = worst;
    stats[1] = t.tscale;
  }
  return MAC_OK;
}

static int train(Net& t, int steps, int batch, float lr, uint64_t seed, float* losses, cudaStream_t st) {
  if (!t.ds_count || steps < 1 || batch < 1 || batch > 64) return MAC_ERR_INVALID;
  const int s = t.ds_size;
  int rc = ensure_shape(t, batch, s, s, s);
  if (rc) return rc;
  if (steps > t.loss_cap) {
    cudaFree(t.loss_hist);
    t.loss_hist = nullptr;
    t.loss_cap = 0;
    if ((rc = cuda_ok(cudaMalloc((void**)&t.loss_hist, steps * sizeof(double))))) return rc;
    t.loss_cap = steps;
  }
  const size_t V1 = (size_t)s * s * s;
  const dim3 g((unsigned)std::min<size_t>((V1 + 255) / 256, 296), batch);
  for (int k = 0; k < steps && !rc; ++k) {
    k_gather_batch<<<g, 256, 0, st>>>(t.ds_r, t.ds_e, t.ds_m, t.ds_count, V1, seed, (uint64_t)k, t.r, t.e, t.m);
    ++t.launches;
    rc = loss_grad(t, t.loss_hist + k, st);
    adam(t, lr, st);
  }
  if (!rc) rc = check_err(t, st);
  if (!rc && losses) {
    std::vector<double> h(steps);
    rc = cuda_ok(cudaMemcpy(h.data(), t.loss_hist, steps * sizeof(double), cudaMemcpyDeviceToHost));
    for (int k = 0; k < steps; ++k) losses[k] = (float)h[k];
  }
  return rc;
}

}  // namespace unet
}  // namespace mac

using mac::unet::Net;

extern "C" {

int mac_unet_create(int device, void** net) {
  if (!net) return MAC_ERR_INVALID;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return MAC_ERR_NO_DEVICE;
  Net* t = nullptr;
  int rc = mac::unet::create(device, &t);
  *net = rc ? nullptr : t;
  return rc;
}

int mac_unet_destroy(void* net) {
  mac::unet::destroy((Net*)net);
  return MAC_OK;
}

int mac_unet_nparams(void* net, int64_t* n) {
  if (!net || !n) return MAC_ERR_INVALID;
  *n = (int64_t)((Net*)net)->np;
  return MAC_OK;
}

int mac_unet_init(void* net, uint64_t seed) {
  Net* t = (Net*)net;
  if (!t) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  std::vector<float> p = mac::unet::init_params(*t, seed);
  return mac::unet::set_params(*t, p.data(), 0);
}

int mac_unet_get_params(void* net, float* host, float* tscale) {
  Net* t = (Net*)net;
  if (!t || !host) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  if (tscale) *tscale = t->tscale;
  return mac::unet::cuda_ok(cudaMemcpy(host, t->p, t->np * 4, cudaMemcpyDeviceToHost));
}

int mac_unet_set_params(void* net, const float* host, float tscale) {
  Net* t = (Net*)net;
  if (!t || !host || !(tscale > 0)) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  t->tscale = tscale;
  return mac::unet::set_params(*t, host, 0);
}

int mac_unet_forward(void* net, int n, int d, int h, int w, const float* r, const int8_t* mask, float* out) {
  Net* t = (Net*)net;
  if (!t || !r || !mask || !out) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  int rc = mac::unet::ensure_shape(*t, n, d, h, w);
  if (rc) return rc;
  const size_t v0 = (size_t)n * d * h * w;
  cudaMemcpy(t->r, r, v0 * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(t->m, mask, v0, cudaMemcpyHostToDevice);
  rc = mac::unet::apply(t, 0);
  if (!rc) rc = mac::unet::check_err(*t, 0);
  if (!rc) rc = mac::unet::cuda_ok(cudaMemcpy(out, t->e, v0 * 4, cudaMemcpyDeviceToHost));
  return rc;
}

int mac_unet_loss_grad(void* net, int n, int d, int h, int w, const float* r, const int8_t* mask, const float* e,
                       double* loss, float* grad) {
  Net* t = (Net*)net;
  if (!t || !r || !mask || !e) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  int rc = mac::unet::ensure_shape(*t, n, d, h, w);
  if (rc) return rc;
  const size_t v0 = (size_t)n * d * h * w;
  cudaMemcpy(t->r, r, v0 * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(t->m, mask, v0, cudaMemcpyHostToDevice);
  cudaMemcpy(t->e, e, v0 * 4, cudaMemcpyHostToDevice);
  rc = mac::unet::loss_grad(*t, t->loss, 0);
  if (!rc) rc = mac::unet::check_err(*t, 0);
  if (!rc && loss) rc = mac::unet::cuda_ok(cudaMemcpy(loss, t->loss, sizeof(double), cudaMemcpyDeviceToHost));
  if (!rc && grad) rc = mac::unet::cuda_ok(cudaMemcpy(grad, t->g, t->np * 4, cudaMemcpyDeviceToHost));
  return rc;
}

int mac_unet_adam_step(void* net, const float* grad, float lr) {
  Net* t = (Net*)net;
  if (!t || !grad) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  int rc = mac::unet::cuda_ok(cudaMemcpy(t->g, grad, t->np * 4, cudaMemcpyHostToDevice));
  if (rc) return rc;
  mac::unet::adam(*t, lr, 0);
  return mac::unet::cuda_ok(cudaDeviceSynchronize());
}

int mac_unet_make_dataset(void* net, int nmasks, int size, int nsnap, int niter, uint64_t seed, double* stats) {
  Net* t = (Net*)net;
  if (!t) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  return mac::unet::make_dataset(*t, nmasks, size, nsnap, niter, seed, stats, 0);
}

int mac_unet_make_dataset_ext(void* net, int nmasks, int size, int nsnap, int niter, uint64_t seed,
                              const int8_t* masks, int nmasks_given, double* stats) {
  Net* t = (Net*)net;
  if (!t || nmasks_given < 0 || nmasks_given > nmasks || (nmasks_given > 0 && !masks)) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  return mac::unet::make_dataset(*t, nmasks, size, nsnap, niter, seed, stats, 0, masks, nmasks_given);
}

int mac_unet_get_sample(void* net, int index, float* r, float* e, int8_t* mask) {
  Net* t = (Net*)net;
  if (!t || index < 0 || index >= t->ds_count) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  const size_t V1 = (size_t)t->ds_size * t->ds_size * t->ds_size;
  int rc = MAC_OK;
  if (r) rc = mac::unet::cuda_ok(cudaMemcpy(r, t->ds_r + index * V1, V1 * 4, cudaMemcpyDeviceToHost));
  if (!rc && e) rc = mac::unet::cuda_ok(cudaMemcpy(e, t->ds_e + index * V1, V1 * 4, cudaMemcpyDeviceToHost));
  if (!rc && mask) rc = mac::unet::cuda_ok(cudaMemcpy(mask, t->ds_m + index * V1, V1, cudaMemcpyDeviceToHost));
  return rc;
}

int mac_unet_train(void* net, int steps, int batch, float lr, uint64_t seed, float* losses) {
  Net* t = (Net*)net;
  if (!t) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  return mac::unet::train(*t, steps, batch, lr, seed, losses, 0);
}

int mac_unet_set_conv(void* net, int staged) {
  Net* t = (Net*)net;
  if (!t || (staged != 0 && staged != 1)) return MAC_ERR_INVALID;
  t->staged_conv = staged;
  return MAC_OK;
}

int mac_unet_time_forward(void* net, int n, int d, int h, int w, int reps, double* ms, double* flops) {
  Net* t = (Net*)net;
  if (!t || reps < 1 || !ms || !flops) return MAC_ERR_INVALID;
  cudaSetDevice(t->device);
  int rc = mac::unet::ensure_shape(*t, n, d, h, w);
  if (rc) return rc;
  const size_t v0 = (size_t)n * d * h * w;
  // a smooth-ish residual on an all-fluid grid: the timing does not depend on the values
  cudaMemset(t->r, 0, v0 * 4);
  cudaMemset(t->m, 1, v0);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  rc = mac::unet::apply(t, 0);
  cudaEventRecord(e0, 0);
  for (int k = 0; k < reps && !rc; ++k) rc = mac::unet::apply(t, 0);
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  float f = 0;
  cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = mac::unet::check_err(*t, 0);
  *ms = f / reps;
  // algorithmic FLOPs: 2 * taps * cin * cout per output voxel over the real (unpadded) channels
  double fl = 0;
  for (int l = 0; l < mac::unet::kNumLayers; ++l) {
    const auto& L = mac::unet::kLayers[l];
    const int lvl = (l <= 1 || l >= 10) ? 0 : ((l <= 3 || l == 7 || l == 8 || l == 9) ? 1 : 2);
    fl += 2.0 * L.taps * L.real_cin * L.real_cout * (double)v0 / (double)(1 << (3 * lvl));
  }
  *flops = fl;
  return rc;
}

int mac_unet_set_loss(void* net, int kind) {
  if (!net || kind < 0 || kind > 1) return MAC_ERR_INVALID;
  ((Net*)net)->loss_kind = kind;
  return MAC_OK;
}

int mac_unet_launch_count(void* net, int64_t* count) {
  if (!net || !count) return MAC_ERR_INVALID;
  *count = ((Net*)net)->launches;
  return MAC_OK;
}

}  // extern "C"

namespace mac {
namespace unet {
int stage(Net* t, int n, int d, int h, int w, float** r, int8_t** m, float** z) {
  int rc = ensure_shape(*t, n, d, h, w);
  if (rc) return rc;
  *r = t->r;
  *m = t->m;
  *z = t->e;
  return MAC_OK;
}
}  // namespace unet
}  // namespace mac

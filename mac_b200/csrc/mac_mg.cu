// Multigrid preconditioner of the pressure solve.
//
// Hierarchy (Galerkin products with piecewise-constant transfer, each level's
// operator scaled by the context's coarse scale; stored as three left-face weights, the
// diagonal, its inverse and the Dirichlet part of the diagonal per cell):
//   level 0  the fine cells of every brick that holds an in-domain cell
//            (8^3 per brick; operator from the per-cell face classes),
//   level 1  4^3 per brick, level 2  2^3 per brick (brick-local, neighbours
//            through the brick neighbour table),
//   level 3  one cell per brick on a dense grid over the bounding box of the
//            domain bricks, levels 4.. dense coarsenings of it.
// Smoother: weighted Jacobi (two sweeps before and after the coarse
// correction); the levels from 4 down are solved by one thread block in
// shared memory, the coarsest (at most 64 cells) exactly with an inverse built
// at set-up. T is the storage and arithmetic type of every level: double
// (plain form) or float (mixed form); the fine residual r and the
// preconditioned residual z the CG iteration exchanges stay double.
#include <cstdio>
#include <cstring>
#include <utility>

#include "mac_internal.cuh"

namespace mac {

// Smoother weights and the per-level scale of the Galerkin operator
// (piecewise-constant transfer over-weights the coarse operator) come from the
// context (Params::mgw1/mgw2/mgws, Ctx::mg_scale; mac_set_smoother). Two
// sweeps with weights w1, w2 damp the error of an eigenvalue lambda of D^-1 A
// (in (0, 2] here: the operators are diagonally dominant) by
// (1 - w1 lambda)(1 - w2 lambda); the V-cycle stays symmetric positive
// definite while that product stays inside (-1, 1) on (0, 2].
constexpr int kCoarsestSweeps = 40;

// Level-1 parent of level-0 cell n (pool index).
__device__ inline int64_t parent1(int64_t n) {
  int o = (int)(n & 511);
  return (n >> 9) * 64 + ((o & 7) >> 1) + 4 * (((o >> 3) & 7) >> 1) + 16 * ((o >> 6) >> 1);
}

// Coordinates of cell i of an nx x ny x nz grid of n cells. Below 2^24 cells
// the quotients come from float reciprocals with one exact correction step
// each (the product's error stays under one unit there); larger grids divide
// in 64 bits.
__device__ inline int qdiv(int i, int d, float rd) {
  int q = (int)((float)i * rd);
  const int r = i - q * d;
  if (r < 0) --q;
  else if (r >= d) ++q;
  return q;
}
__device__ inline void coords3(int64_t i, int nx, int ny, int64_t n, int& x, int& y, int& z) {
  if (n < (int64_t)(1 << 24)) {
    const int ii = (int)i;
    const int xy = qdiv(ii, nx, 1.0f / (float)nx);
    x = ii - xy * nx;
    z = qdiv(xy, ny, 1.0f / (float)ny);
    y = xy - z * ny;
  } else {
    const int64_t xy = i / nx;
    x = (int)(i - xy * nx);
    z = (int)(xy / ny);
    y = (int)(xy - (int64_t)z * ny);
  }
}

// ---------------------------------------------------------------- level 0
// The level-0 sweeps wait mostly on memory latency; in the FP32 form their
// register caps let 16 blocks of 128 threads share an SM without spills (the
// FP64 pre-sweep takes 12; the FP64 post-sweeps would spill under any cap).
// Two Jacobi sweeps from zero, fused: e1 = w D^-1 r, e = e1 + w D^-1 (r - M e1)
// = w D^-1 ((2 - w) r + sum_f ih2_f e1(n_f)).
// With update (every CG iteration but the first) the kernel first finishes
// the previous iteration over all cells of the brick: x += alpha p and
// r = rin - alpha q into rout with the block's partial r.r. rout is not rin,
// so a block staging its face halos reads the old r of its neighbours and
// forms their new r on the fly with the same expression.
template <class T>
__global__ void __launch_bounds__(kBT, sizeof(T) == 4 ? 16 : 12) k0_pre(const int* __restrict__ drow,
                                              const uint16_t* __restrict__ fmask, const double* __restrict__ rin,
                                              double* __restrict__ rout, double* __restrict__ x,
                                              const double* __restrict__ p, const double* __restrict__ q,
                                              double* partial, const Scalars* ds, int update, T* __restrict__ e,
                                              Params P) {
  __shared__ int64_t sb[6];
  __shared__ T sr[kS1];  // w D^-1 r of the brick and its face halo
  const T om = (T)P.mgw1, om2 = (T)P.mgw2, c0 = (T)(P.mgw1 + P.mgw2 - P.mgw1 * P.mgw2);
  const T ih2[3] = {(T)P.ih2[0], (T)P.ih2[1], (T)P.ih2[2]};
  // prologue (static): brick, face neighbours, face masks; each thread takes
  // the z-run of four cells ob + 64 k (its z neighbours' staged values then
  // come from registers in the stencil pass)
  const int b = load_drow(drow, sb);
  const int ob = zrun_base();
  uint16_t mk[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) mk[k] = fmask[(int64_t)b * kCells + ob + 64 * k];
  pdl_entry();
  if (solve_done(&ds->done)) return;
  const double al = update ? ds->alpha : 0.0;
  const int si0 = s1_of(ob);
  double rv[kCPT];
  T srv[kCPT];
  double rr = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int64_t c = (int64_t)b * kCells + ob + 64 * k;
    double v = rin[c];
    if (update) {
      v = v - al * q[c];
      rout[c] = v;
      x[c] += al * p[c];
      rr += v * v;
    }
    rv[k] = v;
    srv[k] = om * (T)P.dtab[active_index(mk[k])] * (T)v;
    sr[si0 + 100 * k] = srv[k];
  }
  __syncthreads();
  stage_h1_halo(sr, sb, [&](int64_t i) {
    const double v = update ? rin[i] - al * q[i] : rin[i];
    return om * (T)P.dtab[active_index(fmask[i])] * (T)v;
  });
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int64_t c = (int64_t)b * kCells + ob + 64 * k;
    const uint16_t m = mk[k];
    T out = 0;
    if (m & kDomainBit) {
      const int si = si0 + 100 * k;
      const T dinv = (T)P.dtab[active_index(m)];
      T s = 0;
#pragma unroll
      for (int f = 0; f < 6; ++f)
        if (m & (1u << f)) s += ih2[f >> 1] * zrun_nbr(sr, srv, si, k, f);
      out = dinv * (c0 * (T)rv[k] + om2 * s);
    }
    e[c] = out;
  }
  if (update) block_sum<kBT>(rr, 0.0, partial);
}

// res = r - M e on the brick, summed over 2x2x2 children into level 1.
template <class T>
__global__ void __launch_bounds__(kBT) k0_restrict(const int* __restrict__ drow,
                                                   const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                                   const T* __restrict__ e, T* __restrict__ r1, Params P,
                                                   const int32_t* __restrict__ done) {
  __shared__ int64_t sb[6];
  __shared__ T se[kS1];
  const T ih2[3] = {(T)P.ih2[0], (T)P.ih2[1], (T)P.ih2[2]};
  // prologue: brick, face neighbours, face masks (static) and r (written by
  // the V-cycle's first kernel, two launches back)
  const int b = load_drow(drow, sb);
  // the stencil pass takes a z-run of four cells of one column per thread
  // (cells zrun_base() + 64 k): z neighbours inside the run from registers
  const int ob = zrun_base();
  uint16_t mk[kCPT];
  double rk[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int64_t c = (int64_t)b * kCells + ob + 64 * k;
    mk[k] = fmask[c];
    rk[k] = r[c];
  }
  pdl_entry();
  if (solve_done(done)) return;
  __syncthreads();
  stage_arr(se, e, b, sb);
  __syncthreads();
  const int si0 = s1_of(ob);
  T ecs[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) ecs[k] = se[si0 + 100 * k];
  T v[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const uint16_t m = mk[k];
    v[k] = 0;
    if (m & kDomainBit) {
      const int si = si0 + 100 * k;
      const T ec = ecs[k];
      T me = 0;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (m & (1u << (8 + f))) me += ih2[f >> 1] * ec;
        if (m & (1u << f)) me -= ih2[f >> 1] * zrun_nbr(se, ecs, si, k, f);
      }
      v[k] = (T)rk[k] - me;
    }
  }
  // the 2x2x2 children of a level-1 cell: z pairs inside the thread's run,
  // x pairs on lanes t, t ^ 1 and y pairs on lanes t, t ^ 8 (x = t & 7,
  // y = (t >> 3) & 7); the lane with x and y even holds the sums
  T s0 = v[0] + v[1], s1 = v[2] + v[3];
  s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
  s0 += __shfl_xor_sync(0xffffffffu, s0, 8);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 8);
  const int x = threadIdx.x & 7, y = (threadIdx.x >> 3) & 7, zh = threadIdx.x >> 6;
  if (!((x | y) & 1)) {
    const size_t base = (size_t)b * 64 + (x >> 1) + 4 * (y >> 1) + 16 * (2 * zh);
    r1[base] = s0;
    r1[base + 16] = s1;
  }
}

// Level-1 parent (within its brick's 64) of cell `off` of a level-0 brick.
__device__ inline int parent_off(int off) { return ((off & 7) >> 1) + 4 * (((off >> 3) & 7) >> 1) + 16 * (off >> 7); }

// Post-smoothing at level 0. FIRST: ep = e + P e1 (coarse correction added on
// the fly, the level-1 parent of every staged cell read as it is staged), out
// = ep + w D^-1 (r - M ep) into eout. Otherwise a plain sweep writing the FP64
// preconditioned residual z and the block's partial r.z. The cells' r and
// face masks are loaded first, so they are in flight during the staging.
template <class T, bool FIRST>
__global__ void __launch_bounds__(kBT, sizeof(T) == 4 ? 16 : 1) k0_post(const int* __restrict__ drow,
                                               const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                               const T* __restrict__ e, const T* __restrict__ e1, T* __restrict__ eout,
                                               double* __restrict__ z, double* partial, Params P,
                                               const int32_t* __restrict__ done) {
  __shared__ int64_t sb[6];
  __shared__ T se[kS1];  // e (plus the coarse correction when FIRST) with face halo
  const T om = (T)(FIRST ? P.mgw1 : P.mgw2), ih2[3] = {(T)P.ih2[0], (T)P.ih2[1], (T)P.ih2[2]};
  // prologue: brick, face neighbours, face masks (static), r and, when FIRST,
  // the brick's pre-smoothed e (both written many launches back)
  const int b = load_drow(drow, sb);
  const int ob = zrun_base();  // the stencil pass's z-run (cells ob + 64 k)
  uint16_t mk[kCPT];
  double rk[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int64_t c = (int64_t)b * kCells + ob + 64 * k;
    mk[k] = fmask[c];
    rk[k] = r[c];
  }
  T v[4];
  if (FIRST) load4(e + (int64_t)b * kCells + 4 * threadIdx.x, v);
  pdl_entry();
  if (solve_done(done)) return;
  if (FIRST) {
    // the brick: cells 4t..4t+3 of one row share two level-1 parents
    const int o4 = 4 * threadIdx.x;
    const int p0 = parent_off(o4);
    const T c0 = e1[(size_t)b * 64 + p0], c1 = e1[(size_t)b * 64 + p0 + 1];
    __syncthreads();
    stage_h1_halo(se, sb, [&](int64_t i) { return e[i] + e1[(i >> 9) * 64 + parent_off((int)(i & 511))]; });
    const int si = s1_of(o4);
    se[si] = v[0] + c0;
    se[si + 1] = v[1] + c0;
    se[si + 2] = v[2] + c1;
    se[si + 3] = v[3] + c1;
  } else {
    __syncthreads();
    stage_arr(se, e, b, sb);
  }
  __syncthreads();
  const int si0 = s1_of(ob);
  T eps[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) eps[k] = se[si0 + 100 * k];
  double rz = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int64_t c = (int64_t)b * kCells + ob + 64 * k;
    const uint16_t m = mk[k];
    if (!(m & kDomainBit)) {
      if (FIRST) eout[c] = (T)0;
      else z[c] = 0.0;
      continue;
    }
    const int si = si0 + 100 * k;
    const T epc = eps[k];
    T me = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (m & (1u << (8 + f))) me += ih2[f >> 1] * epc;
      if (m & (1u << f)) me -= ih2[f >> 1] * zrun_nbr(se, eps, si, k, f);
    }
    double rc = rk[k];
    T out = epc + om * (T)P.dtab[active_index(m)] * ((T)rc - me);
    if (FIRST) {
      eout[c] = out;
    } else {
      z[c] = (double)out;
      rz += rc * (double)out;
    }
  }
  if (!FIRST) block_sum<kBT>(rz, 0.0, partial);
}

// ---- level 0 with one sweep before and after the coarse correction.
// Pre-sweep, residual and restriction in one pass: with e = w D^-1 r (one
// Jacobi sweep from zero, pointwise) the residual r - M e needs only the
// staged w D^-1 r of the brick and its face halo, which k0_pre's staging
// already forms; the sum over 2x2x2 children goes to level 1. e is not
// stored: the post-sweep recomputes it from r. The CG update is folded in as
// in k0_pre.
template <class T>
__global__ void __launch_bounds__(kBT, sizeof(T) == 4 ? 16 : 12) k0_pre_restrict(
    const int* __restrict__ drow, const uint16_t* __restrict__ fmask,
    const double* __restrict__ rin, double* __restrict__ rout, double* __restrict__ x, const double* __restrict__ p,
    const double* __restrict__ q, double* partial, const Scalars* ds, int update, T* __restrict__ r1, Params P) {
  pdl_entry();
  if (solve_done(&ds->done)) return;
  __shared__ int64_t sb[6];
  __shared__ T sr[kS1];    // e = w D^-1 r of the brick and its face halo
  __shared__ T res[kCells];
  const T om = (T)P.mgws, ih2[3] = {(T)P.ih2[0], (T)P.ih2[1], (T)P.ih2[2]};
  const double al = update ? ds->alpha : 0.0;
  const int b = load_drow(drow, sb);
  double rv[kCPT];
  uint16_t mk[kCPT];
  double rr = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int o = threadIdx.x + kBT * k;
    const int64_t c = (int64_t)b * kCells + o;
    double v = rin[c];
    if (update) {
      v = v - al * q[c];
      rout[c] = v;
      x[c] += al * p[c];
      rr += v * v;
    }
    rv[k] = v;
    const uint16_t m = fmask[c];
    mk[k] = m;
    sr[s1_of(o)] = om * (T)P.dtab[active_index(m)] * (T)v;
  }
  __syncthreads();
  stage_h1_halo(sr, sb, [&](int64_t i) {
    const double v = update ? rin[i] - al * q[i] : rin[i];
    return om * (T)P.dtab[active_index(fmask[i])] * (T)v;
  });
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int o = threadIdx.x + kBT * k;
    const uint16_t m = mk[k];
    T v = 0;
    if (m & kDomainBit) {
      const int si = s1_of(o);
      const T ec = sr[si];
      T me = 0;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (m & (1u << (8 + f))) me += ih2[f >> 1] * ec;
        if (m & (1u << f)) me -= ih2[f >> 1] * sr[si + s1_off(f)];
      }
      v = (T)rv[k] - me;
    }
    res[o] = v;
  }
  __syncthreads();
  const int o = threadIdx.x;
  if (o < 64) {
    const int X = o & 3, Y = (o >> 2) & 3, Z = o >> 4;
    const int base = 2 * X + 16 * Y + 128 * Z;
    r1[(size_t)b * 64 + o] = res[base] + res[base + 1] + res[base + 8] + res[base + 9] + res[base + 64] +
                             res[base + 65] + res[base + 72] + res[base + 73];
  }
  if (update) block_sum<kBT>(rr, 0.0, partial);
}

// The one post-sweep: ep = w D^-1 r + P e1 (pre-sweep recomputed, coarse
// correction added, on the brick and its face halo), z = ep + w D^-1 (r - M ep)
// in FP64 with the block's partial r.z.
template <class T>
__global__ void __launch_bounds__(kBT, sizeof(T) == 4 ? 12 : 1) k0_post_one(
    const int* __restrict__ drow, const uint16_t* __restrict__ fmask,
    const double* __restrict__ r, const T* __restrict__ e1, double* __restrict__ z, double* partial, Params P,
    const int32_t* __restrict__ done) {
  pdl_entry();
  if (solve_done(done)) return;
  __shared__ int64_t sb[6];
  __shared__ T se[kS1];
  const T om = (T)P.mgws, ih2[3] = {(T)P.ih2[0], (T)P.ih2[1], (T)P.ih2[2]};
  const int b = load_drow(drow, sb);
  uint16_t mk[kCPT];
  double rk[kCPT];
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int o = threadIdx.x + kBT * k;
    const int64_t c = (int64_t)b * kCells + o;
    mk[k] = fmask[c];
    rk[k] = r[c];
    se[s1_of(o)] = om * (T)P.dtab[active_index(mk[k])] * (T)rk[k] + e1[(size_t)b * 64 + parent_off(o)];
  }
  __syncthreads();
  stage_h1_halo(se, sb, [&](int64_t i) {
    return om * (T)P.dtab[active_index(fmask[i])] * (T)r[i] + e1[(i >> 9) * 64 + parent_off((int)(i & 511))];
  });
  __syncthreads();
  double rz = 0;
#pragma unroll
  for (int k = 0; k < kCPT; ++k) {
    const int o = threadIdx.x + kBT * k;
    const int64_t c = (int64_t)b * kCells + o;
    const uint16_t m = mk[k];
    if (!(m & kDomainBit)) {
      z[c] = 0.0;
      continue;
    }
    const int si = s1_of(o);
    const T epc = se[si];
    T me = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (m & (1u << (8 + f))) me += ih2[f >> 1] * epc;
      if (m & (1u << f)) me -= ih2[f >> 1] * se[si + s1_off(f)];
    }
    const double rc = rk[k];
    const T out = epc + om * (T)P.dtab[active_index(m)] * ((T)rc - me);
    z[c] = (double)out;
    rz += rc * (double)out;
  }
  block_sum<kBT>(rz, 0.0, partial);
}

// ---- the V-cycle's first kernel with the bricks prefetched asynchronously.
// A block walks the domain bricks j = blockIdx.x, blockIdx.x + G, ... (G
// blocks resident on all SMs at once). While it works on one brick, one
// thread has the next brick's CG vectors r, q, x, p (4 KB each, FP64) and its
// face classes (1 KB) in flight into the other half of a two-stage shared
// buffer: five cp.async.bulk copies completing on the stage's mbarrier. The
// face halos are read with plain loads. The arithmetic is k0_pre's (two
// sweeps, RESTRICT = false) or k0_pre_restrict's (one sweep with the residual
// restricted to level 1, RESTRICT = true), value for value; only the block
// partials of r.r sum several bricks. Every wait is bounded: a wait that runs
// out sets kErrTimeout, waits once more for the copies in flight and returns.
namespace bulk {
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
// global -> shared, 16-byte aligned addresses, size a multiple of 16
__device__ __forceinline__ void copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   saddr(dst)),
               "l"(src), "r"(bytes), "r"(saddr(bar))
               : "memory");
}
__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool wait(uint64_t* bar, uint32_t parity) {
  for (int i = 0; i < (1 << 20); ++i)
    if (try_wait(bar, parity)) return true;
  return false;
}
}  // namespace bulk

constexpr int kBulkVec = kCells * 8;                   // one FP64 vector of a brick
constexpr int kBulkStage = 4 * kBulkVec + kCells * 2;  // r, q, x, p and the face classes

template <class T>
constexpr int bulk_smem() {
  return 2 * kBulkStage + kS1 * (int)sizeof(T) + kCells * (int)sizeof(T);
}

template <class T, bool RESTRICT>
__global__ void __launch_bounds__(kBT) k0_head_bulk(const int* __restrict__ dbl, int nd, const int* __restrict__ nbr,
                                                    const uint16_t* __restrict__ fmask, const double* __restrict__ rin,
                                                    double* __restrict__ rout, double* __restrict__ x,
                                                    const double* __restrict__ p, const double* __restrict__ q,
                                                    double* partial, Scalars* ds, int update, T* __restrict__ e,
                                                    T* __restrict__ r1, Params P) {
  pdl_entry();
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ int64_t sb[6];
  __shared__ __align__(8) uint64_t full[2];
  __shared__ int failed;
  if (solve_done(&ds->done)) return;
  T* sr = reinterpret_cast<T*>(smem + 2 * kBulkStage);  // w D^-1 r (brick and face halo)
  T* res = sr + kS1;                                     // RESTRICT: the brick's residual
  const int tid = threadIdx.x;
  const T om = (T)(RESTRICT ? P.mgws : P.mgw1), om2 = (T)P.mgw2, c0 = (T)(P.mgw1 + P.mgw2 - P.mgw1 * P.mgw2), ih2[3] = {(T)P.ih2[0], (T)P.ih2[1], (T)P.ih2[2]};
  const double al = update ? ds->alpha : 0.0;
  const uint32_t bytes = update ? (uint32_t)kBulkStage : (uint32_t)(kBulkVec + kCells * 2);
  auto issue = [&](int j, int st) {
    const int64_t base = (int64_t)dbl[j] * kCells;
    uint8_t* s = smem + st * kBulkStage;
    bulk::expect_tx(&full[st], bytes);
    bulk::copy(s, rin + base, kBulkVec, &full[st]);
    if (update) {
      bulk::copy(s + kBulkVec, q + base, kBulkVec, &full[st]);
      bulk::copy(s + 2 * kBulkVec, x + base, kBulkVec, &full[st]);
      bulk::copy(s + 3 * kBulkVec, p + base, kBulkVec, &full[st]);
    }
    bulk::copy(s + 4 * kBulkVec, fmask + base, kCells * 2, &full[st]);
  };
  if (tid == 0) {
    bulk::mbar_init(&full[0]);
    bulk::mbar_init(&full[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    failed = 0;
  }
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < nd) issue(blockIdx.x, 0);
  double rr = 0;
  int it = 0;
  bool next_issued = false;  // a copy into the other stage is in flight
  for (int j = blockIdx.x; j < nd; j += gridDim.x, ++it) {
    const int st = it & 1;
    const int b = dbl[j];
    load_face_bases(nbr, b, sb);
    next_issued = j + (int)gridDim.x < nd;
    if (tid == 0 && next_issued) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(j + gridDim.x, st ^ 1);
    }
    __syncthreads();
    // the face halos with plain loads, all in flight before any store
    stage_h1_halo(sr, sb, [&](int64_t i) {
      const double v = update ? rin[i] - al * q[i] : rin[i];
      return om * (T)P.dtab[active_index(fmask[i])] * (T)v;
    });
    if (!bulk::wait(&full[st], (uint32_t)((it >> 1) & 1))) {
      atomicOr(&ds->err, kErrTimeout);
      failed = 1;
    }
    __syncthreads();
    if (failed) break;
    const double* sR = reinterpret_cast<const double*>(smem + st * kBulkStage);
    const double* sQ = sR + kCells;
    const double* sX = sR + 2 * kCells;
    const double* sP = sR + 3 * kCells;
    const uint16_t* sM = reinterpret_cast<const uint16_t*>(sR + 4 * kCells);
    double rv[kCPT];
    uint16_t mk[kCPT];
#pragma unroll
    for (int k = 0; k < kCPT; ++k) {
      const int o = tid + kBT * k;
      const int64_t c = (int64_t)b * kCells + o;
      double v = sR[o];
      if (update) {
        v = v - al * sQ[o];
        rout[c] = v;
        x[c] = sX[o] + al * sP[o];
        rr += v * v;
      }
      rv[k] = v;
      const uint16_t m = sM[o];
      mk[k] = m;
      sr[s1_of(o)] = om * (T)P.dtab[active_index(m)] * (T)v;
    }
    __syncthreads();
    if (RESTRICT) {
#pragma unroll
      for (int k = 0; k < kCPT; ++k) {
        const int o = tid + kBT * k;
        const uint16_t m = mk[k];
        T v = 0;
        if (m & kDomainBit) {
          const int si = s1_of(o);
          const T ec = sr[si];
          T me = 0;
#pragma unroll
          for (int f = 0; f < 6; ++f) {
            if (m & (1u << (8 + f))) me += ih2[f >> 1] * ec;
            if (m & (1u << f)) me -= ih2[f >> 1] * sr[si + s1_off(f)];
          }
          v = (T)rv[k] - me;
        }
        res[o] = v;
      }
      __syncthreads();
      if (tid < 64) {
        const int X = tid & 3, Y = (tid >> 2) & 3, Z = tid >> 4;
        const int base = 2 * X + 16 * Y + 128 * Z;
        r1[(size_t)b * 64 + tid] = res[base] + res[base + 1] + res[base + 8] + res[base + 9] + res[base + 64] +
                                   res[base + 65] + res[base + 72] + res[base + 73];
      }
    } else {
#pragma unroll
      for (int k = 0; k < kCPT; ++k) {
        const int o = tid + kBT * k;
        const int64_t c = (int64_t)b * kCells + o;
        const uint16_t m = mk[k];
        T out = 0;
        if (m & kDomainBit) {
          const int si = s1_of(o);
          const T dinv = (T)P.dtab[active_index(m)];
          T s = 0;
#pragma unroll
          for (int f = 0; f < 6; ++f)
            if (m & (1u << f)) s += ih2[f >> 1] * sr[si + s1_off(f)];
          out = dinv * (c0 * (T)rv[k] + om2 * s);
        }
        e[c] = out;
      }
    }
    __syncthreads();
  }
  if (failed) {
    // the copies of this brick and of the next may still be in flight: wait
    // for them (bounded) before the block's shared memory is given up
    const int st = it & 1;
    if (tid == 0) {
      bulk::wait(&full[st], (uint32_t)((it >> 1) & 1));
      if (next_issued) bulk::wait(&full[st ^ 1], (uint32_t)(((it + 1) >> 1) & 1));
    }
    return;
  }
  if (update) block_sum<kBT>(rr, 0.0, partial);
}

// ------------------------------------------------------- levels 1, 2 (bricks)
template <int D>
__device__ inline int64_t lidx(const int* __restrict__ nbr, int b, int x, int y, int z) {
  int dx = x < 0 ? -1 : (x >= D ? 1 : 0);
  int dy = y < 0 ? -1 : (y >= D ? 1 : 0);
  int dz = z < 0 ? -1 : (z >= D ? 1 : 0);
  int nb = ((dx | dy | dz) == 0) ? b : nbr[(size_t)b * kNbr + nbr_index(dx, dy, dz)];
  if (nb < 0) return -1;
  return (int64_t)nb * (D * D * D) + (x - D * dx) + D * (y - D * dy) + D * D * (z - D * dz);
}

// Brick-level kernels run 256 threads over 256 / D^3 bricks; the bricks and
// their six face neighbours are read once per block into shared memory, so no
// thread chains a brick-table load before its own loads.
template <int D>
struct LBricks {
  static constexpr int N = D * D * D;
  static constexpr int BPB = 256 / N;  // bricks per block
};

// sbr[7 * j + k]: local brick j's pool index (k = 0) and its face neighbours
// -x, +x, -y, +y, -z, +z (k = 1..6), -1 when absent or past the list.
template <int D>
__device__ inline void load_lbricks(const int* __restrict__ drow, int nd, int* sbr) {
  constexpr int BPB = LBricks<D>::BPB;
  for (int t = threadIdx.x; t < 7 * BPB; t += blockDim.x) {
    const int j = t / 7, k = t % 7;
    const int gb = blockIdx.x * BPB + j;
    sbr[t] = gb < nd ? drow[8 * (size_t)gb + k] : -1;
  }
}

// Weights w: 6 slots of ncap entries: [0..2] left faces, [3] diagonal, [4] inverse, [5] Dirichlet part.
// The six neighbour indices of cell (x, y, z) (-1 absent): [2a] = -e_a, [2a+1] = +e_a.
template <int D>
__device__ inline void lnbrs(const int* sb, int x, int y, int z, int64_t* n) {
  constexpr int N = D * D * D;
  const int c[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int pl[3] = {x, y, z}, pr[3] = {x, y, z};
    int kl = 0, kr = 0;
    if (c[a] > 0) pl[a] = c[a] - 1;
    else { kl = 1 + 2 * a; pl[a] = D - 1; }
    if (c[a] < D - 1) pr[a] = c[a] + 1;
    else { kr = 2 + 2 * a; pr[a] = 0; }
    const int bl = sb[kl], br = sb[kr];
    n[2 * a] = bl < 0 ? -1 : (int64_t)bl * N + pl[0] + D * pl[1] + D * D * pl[2];
    n[2 * a + 1] = br < 0 ? -1 : (int64_t)br * N + pr[0] + D * pr[1] + D * D * pr[2];
  }
}

// M e at cell i: every load is issued before any term is tested (a missing
// neighbour reads cell i itself and drops out through its zero weight), then
// the terms are summed in the fixed order.
template <class T, int D>
__device__ inline T apply_l(const T* __restrict__ e, const T* __restrict__ w, size_t ncap,
                                 const int64_t* n, size_t i, T ec) {
  T wl[3], wr[3], el[3], er[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int64_t jl = n[2 * a] < 0 ? (int64_t)i : n[2 * a];
    const int64_t jr = n[2 * a + 1] < 0 ? (int64_t)i : n[2 * a + 1];
    wl[a] = w[a * ncap + i];
    el[a] = e[jl];
    wr[a] = n[2 * a + 1] < 0 ? (T)0 : w[a * ncap + jr];
    er[a] = e[jr];
  }
  T s = w[3 * ncap + i] * ec;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (wl[a] != 0) s -= wl[a] * el[a];
    if (wr[a] != 0) s -= wr[a] * er[a];
  }
  return s;
}

template <class T, int D>
__global__ void __launch_bounds__(256) kl_pre(const int* __restrict__ drow, int nd,
                                              const T* __restrict__ w, size_t ncap, const T* __restrict__ r,
                                              T* __restrict__ e, T w1, T w2, const int32_t* __restrict__ done) {
  constexpr int N = D * D * D;
  __shared__ int sbr[7 * LBricks<D>::BPB];
  // prologue (static): the brick tables, the cell's weights and its
  // neighbours' inverse diagonals
  load_lbricks<D>(drow, nd, sbr);
  __syncthreads();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = g < (int64_t)nd * N;
  size_t i = 0;
  T dinv = 0;
  uint32_t jl[3] = {0, 0, 0}, jr[3] = {0, 0, 0};  // cell indices of a level (below 2^32: 64 per brick)
  T wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0}, dl[3] = {0, 0, 0}, dr[3] = {0, 0, 0};
  if (live) {
    const int* sb = sbr + 7 * (threadIdx.x / N);
    const int o = (int)(g % N);
    i = (size_t)sb[0] * N + o;
    dinv = w[4 * ncap + i];
    const int x = o % D, y = (o / D) % D, z = o / (D * D);
    int64_t n[6];
    lnbrs<D>(sb, x, y, z, n);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      jl[a] = (uint32_t)(n[2 * a] < 0 ? (int64_t)i : n[2 * a]);
      jr[a] = (uint32_t)(n[2 * a + 1] < 0 ? (int64_t)i : n[2 * a + 1]);
      wl[a] = w[a * ncap + i];
      dl[a] = w[4 * ncap + jl[a]];
      wr[a] = n[2 * a + 1] < 0 ? (T)0 : w[a * ncap + jr[a]];
      dr[a] = w[4 * ncap + jr[a]];
    }
  }
  pdl_entry();
  if (!live || solve_done(done)) return;
  if (dinv == 0) {
    e[i] = (T)0;
    return;
  }
  T rl[3], rr[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    rl[a] = r[jl[a]];
    rr[a] = r[jr[a]];
  }
  T s = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (wl[a] != 0) s += wl[a] * w1 * dl[a] * rl[a];
    if (wr[a] != 0) s += wr[a] * w1 * dr[a] * rr[a];
  }
  e[i] = dinv * ((w1 + w2 - w1 * w2) * r[i] + w2 * s);
}

// Sum over aligned groups of 8 lanes; the result is valid in the group's first lane.
template <class V>
__device__ inline V sum8(V v) {
  v += __shfl_down_sync(0xffffffffu, v, 4, 8);
  v += __shfl_down_sync(0xffffffffu, v, 2, 8);
  v += __shfl_down_sync(0xffffffffu, v, 1, 8);
  return v;
}

// Residual of a brick level summed over children: D = 4 writes level 2
// (brick-local), D = 2 writes the dense level 3 at the brick's position. One
// thread per fine cell, the 8 children of a coarse cell on 8 adjacent lanes.
template <class T, int D>
__global__ void __launch_bounds__(256) kl_restrict(const int* __restrict__ drow, int nd,
                                                   const int* __restrict__ bkey, const T* __restrict__ w, size_t ncap,
                                                   const T* __restrict__ r, const T* __restrict__ e, T* __restrict__ rc,
                                                   DenseGrid g3, const int32_t* __restrict__ done) {
  constexpr int H = D / 2;
  constexpr int N = D * D * D;
  __shared__ int sbr[7 * LBricks<D>::BPB];
  // prologue: the brick tables and weights (static) and the cell's residual
  // (written two or more launches back)
  load_lbricks<D>(drow, nd, sbr);
  __syncthreads();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = g < (int64_t)nd * N;  // nd * N is a multiple of 8: groups are whole
  const int* sb = sbr + 7 * (threadIdx.x / N);
  int b = 0, p = 0;
  bool act = false;
  size_t i = 0;
  uint32_t jl[3] = {0, 0, 0}, jr[3] = {0, 0, 0};  // cell indices of a level (below 2^32)
  T wd = 0, ri = 0, wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0};
  if (live) {
    b = sb[0];
    const int o = (int)(g % N);
    p = o >> 3;
    const int k = o & 7;
    const int X = p % H, Y = (p / H) % H, Z = p / (H * H);
    const int x = 2 * X + (k & 1), y = 2 * Y + ((k >> 1) & 1), z = 2 * Z + (k >> 2);
    i = (size_t)b * N + x + D * y + D * D * z;
    act = w[4 * ncap + i] != 0;
    if (act) {
      int64_t n[6];
      lnbrs<D>(sb, x, y, z, n);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        jl[a] = (uint32_t)(n[2 * a] < 0 ? (int64_t)i : n[2 * a]);
        jr[a] = (uint32_t)(n[2 * a + 1] < 0 ? (int64_t)i : n[2 * a + 1]);
        wl[a] = w[a * ncap + i];
        wr[a] = n[2 * a + 1] < 0 ? (T)0 : w[a * ncap + jr[a]];
      }
      wd = w[3 * ncap + i];
      ri = r[i];
    }
  }
  pdl_entry();
  if (solve_done(done)) return;
  T v = 0;
  if (act) {
    // r - M e in apply_l's order
    T el[3], er[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      el[a] = e[jl[a]];
      er[a] = e[jr[a]];
    }
    T s = wd * e[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (wl[a] != 0) s -= wl[a] * el[a];
      if (wr[a] != 0) s -= wr[a] * er[a];
    }
    v = ri - s;
  }
  v = sum8(v);
  if (live && (threadIdx.x & 7) == 0) {
    if (D == 2) rc[g3.index(bkey[3 * b], bkey[3 * b + 1], bkey[3 * b + 2])] = (T)v;
    else rc[(size_t)b * H * H * H + p] = (T)v;
  }
}

// One Jacobi sweep at a brick level, optionally adding the coarse correction
// first (D = 4: from level 2 bricks; D = 2: from the dense level 3).
template <class T, int D, bool WITH_COARSE>
__global__ void __launch_bounds__(256) kl_jacobi(const int* __restrict__ drow, int nd,
                                                 const int* __restrict__ bkey, const T* __restrict__ w, size_t ncap,
                                                 const T* __restrict__ r, const T* __restrict__ e,
                                                 const T* __restrict__ ec, T* __restrict__ eout, DenseGrid g3,
                                                 T om, const int32_t* __restrict__ done) {
  constexpr int N = D * D * D;
  constexpr int H = D / 2;
  __shared__ int sbr[7 * LBricks<D>::BPB];
  __shared__ int64_t sdi[7 * LBricks<D>::BPB];  // D = 2: dense level-3 index of each table brick
  // prologue: brick tables and weights (static), r, and with the coarse
  // correction this level's e (both written two or more launches back; e
  // without it is the previous launch's output and waits)
  load_lbricks<D>(drow, nd, sbr);
  __syncthreads();
  if (WITH_COARSE && D == 2) {
    for (int t = threadIdx.x; t < 7 * LBricks<D>::BPB; t += blockDim.x) {
      const int bb = sbr[t];
      sdi[t] = bb < 0 ? 0 : g3.index_or0(bkey[3 * bb], bkey[3 * bb + 1], bkey[3 * bb + 2]);
    }
    __syncthreads();
  }
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = g < (int64_t)nd * N;
  const int* sb = sbr + 7 * (threadIdx.x / N);
  const int o = live ? (int)(g % N) : 0;
  const size_t i = live ? (size_t)sb[0] * N + o : 0;
  const int x = o % D, y = (o / D) % D, z = o / (D * D);
  // stencil points: 0 = the cell, 1 + 2a / 2 + 2a = its -/+ neighbour on axis
  // a (an absent neighbour is the cell itself and drops out through its zero
  // weight): their cell indices ei in this level and, with the coarse
  // correction, ci in the coarser one (32-bit: below 64 cells a brick)
  uint32_t ei[7], ci[7];
  T wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0}, ev[7] = {0, 0, 0, 0, 0, 0, 0};
  T dinv = 0, wd = 0, ri = 0;
  const int jt = 7 * (threadIdx.x / N);  // this brick's row in the tables
  auto point = [&](int q, int k, int px, int py, int pz) {
    const int nb = sb[k];
    ei[q] = (uint32_t)((size_t)nb * N + px + D * py + D * D * pz);
    if (WITH_COARSE) {
      if (D == 2) ci[q] = (uint32_t)sdi[jt + k];
      else ci[q] = (uint32_t)((size_t)nb * H * H * H + (px >> 1) + H * (py >> 1) + H * H * (pz >> 1));
    }
  };
  point(0, 0, x, y, z);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int c[3] = {x, y, z};
    int pl[3] = {x, y, z}, pr[3] = {x, y, z};
    int kl = 0, kr = 0;
    if (c[a] > 0) pl[a] = c[a] - 1;
    else { kl = 1 + 2 * a; pl[a] = D - 1; }
    if (c[a] < D - 1) pr[a] = c[a] + 1;
    else { kr = 2 + 2 * a; pr[a] = 0; }
    const bool hl = sb[kl] >= 0, hr = sb[kr] >= 0;
    if (!hl) { kl = 0; pl[0] = x; pl[1] = y; pl[2] = z; }
    if (!hr) { kr = 0; pr[0] = x; pr[1] = y; pr[2] = z; }
    if (live) {
      point(1 + 2 * a, kl, pl[0], pl[1], pl[2]);
      point(2 + 2 * a, kr, pr[0], pr[1], pr[2]);
      wl[a] = w[a * ncap + i];
      wr[a] = hr ? w[a * ncap + ei[2 + 2 * a]] : (T)0;
    }
  }
  if (live) {
    dinv = w[4 * ncap + i];
    wd = w[3 * ncap + i];
    ri = r[i];
    if (WITH_COARSE) {
#pragma unroll
      for (int q = 0; q < 7; ++q) ev[q] = e[ei[q]];
    }
  }
  pdl_entry();
  if (!live || solve_done(done)) return;
  if (dinv == 0) {
    eout[i] = (T)0;
    return;
  }
  // e plus the coarse correction at each stencil point
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    if (WITH_COARSE) ev[q] += ec[ci[q]];
    else ev[q] = e[ei[q]];
  }
  T s = wd * ev[0];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (wl[a] != 0) s -= wl[a] * ev[1 + 2 * a];
    if (wr[a] != 0) s -= wr[a] * ev[2 + 2 * a];
  }
  eout[i] = ev[0] + om * dinv * (ri - s);
}

// ------------------------------------------------------------ dense levels
// Dense level view: arrays of n cells, weights in 6 slots.
template <class T>
struct DView {
  int nx, ny, nz;
  int64_t n;
  T* e;
  T* e2;
  T* r;
  T* w;  // [6][n]
  T w1, w2;  // smoother weights of the two sweeps
  __device__ int64_t at(int x, int y, int z) const { return x + (int64_t)nx * (y + (int64_t)ny * z); }
};

template <class T>
__device__ inline T dense_apply(const DView<T>& L, const T* e, int64_t i, int x, int y, int z, T ec) {
  int64_t n = L.n;
  T s = L.w[3 * n + i] * ec;
  int c[3] = {x, y, z};
  int dim[3] = {L.nx, L.ny, L.nz};
  int64_t stride[3] = {1, L.nx, (int64_t)L.nx * L.ny};
  for (int a = 0; a < 3; ++a) {
    T wl = L.w[a * n + i];
    if (wl != 0 && c[a] > 0) s -= wl * e[i - stride[a]];
    if (c[a] + 1 < dim[a]) {
      T wr = L.w[a * n + i + stride[a]];
      if (wr != 0) s -= wr * e[i + stride[a]];
    }
  }
  return s;
}

// Device-wide dense kernels for level 3.
template <class T>
__global__ void kd_pre(DView<T> L, const int32_t* __restrict__ done) {
  // prologue (static): the cell's and its neighbours' weights and inverse diagonals
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < L.n;
  const int64_t n = L.n;
  T dinv = 0, wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0}, dl[3] = {0, 0, 0}, dr[3] = {0, 0, 0};
  bool hl[3] = {false, false, false}, hr[3] = {false, false, false};
  int64_t stride[3] = {1, L.nx, (int64_t)L.nx * L.ny};
  if (live) {
    dinv = L.w[4 * n + i];
    int x, y, z;
    coords3(i, L.nx, L.ny, L.n, x, y, z);
    const int c[3] = {x, y, z};
    const int dim[3] = {L.nx, L.ny, L.nz};
    for (int a = 0; a < 3; ++a) {
      wl[a] = L.w[a * n + i];
      hl[a] = wl[a] != 0 && c[a] > 0;
      if (hl[a]) dl[a] = L.w[4 * n + i - stride[a]];
      if (c[a] + 1 < dim[a]) {
        wr[a] = L.w[a * n + i + stride[a]];
        hr[a] = wr[a] != 0;
        if (hr[a]) dr[a] = L.w[4 * n + i + stride[a]];
      }
    }
  }
  pdl_entry();
  if (!live || solve_done(done)) return;
  if (dinv == 0) {
    L.e[i] = (T)0;
    return;
  }
  T s = 0;
  for (int a = 0; a < 3; ++a) {
    if (hl[a]) s += wl[a] * L.w1 * dl[a] * L.r[i - stride[a]];
    if (hr[a]) s += wr[a] * L.w1 * dr[a] * L.r[i + stride[a]];
  }
  L.e[i] = dinv * ((L.w1 + L.w2 - L.w1 * L.w2) * L.r[i] + L.w2 * s);
}

// One thread per (coarse cell, child), the 8 children on adjacent lanes.
template <class T>
__global__ void kd_restrict(DView<T> F, DView<T> C, const int32_t* __restrict__ done) {
  // prologue: weights (static) and the fine residual (written two launches back)
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t I = g >> 3;
  const int k = (int)(g & 7);
  const int64_t n = F.n;
  bool act = false;
  int64_t i = 0;
  int c[3] = {0, 0, 0};
  const int dim[3] = {F.nx, F.ny, F.nz};
  const int64_t stride[3] = {1, F.nx, (int64_t)F.nx * F.ny};
  T wd = 0, ri = 0, wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0};
  if (I < C.n) {
    int X, Y, Z;
    coords3(I, C.nx, C.ny, C.n, X, Y, Z);
    c[0] = 2 * X + (k & 1);
    c[1] = 2 * Y + ((k >> 1) & 1);
    c[2] = 2 * Z + (k >> 2);
    if (c[0] < F.nx && c[1] < F.ny && c[2] < F.nz) {
      i = F.at(c[0], c[1], c[2]);
      act = F.w[4 * n + i] != 0;
      if (act) {
        wd = F.w[3 * n + i];
        ri = F.r[i];
        for (int a = 0; a < 3; ++a) {
          wl[a] = F.w[a * n + i];
          if (c[a] + 1 < dim[a]) wr[a] = F.w[a * n + i + stride[a]];
        }
      }
    }
  }
  pdl_entry();
  if (solve_done(done)) return;
  T s = 0;
  if (act) {
    // r - M e in dense_apply's order
    const T* e = F.e;
    T m = wd * e[i];
    for (int a = 0; a < 3; ++a) {
      if (wl[a] != 0 && c[a] > 0) m -= wl[a] * e[i - stride[a]];
      if (c[a] + 1 < dim[a]) {
        if (wr[a] != 0) m -= wr[a] * e[i + stride[a]];
      }
    }
    s = ri - m;
  }
  s = sum8(s);
  if (I < C.n && k == 0) C.r[I] = (T)s;
}

template <class T, bool WITH_COARSE>
__global__ void kd_jacobi(DView<T> L, const T* __restrict__ ein, T* __restrict__ eout, DView<T> C,
                          const int32_t* __restrict__ done) {
  // prologue: weights (static), r, and with the coarse correction this
  // level's e (written three launches back); without it e is the previous
  // launch's output and waits
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < L.n;
  const int64_t n = L.n;
  int c[3] = {0, 0, 0};
  const int dim[3] = {L.nx, L.ny, L.nz};
  const int64_t stride[3] = {1, L.nx, (int64_t)L.nx * L.ny};
  T dinv = 0, wd = 0, ri = 0, wl[3] = {0, 0, 0}, wr[3] = {0, 0, 0};
  bool hl[3] = {false, false, false}, hr[3] = {false, false, false};
  T vc = 0, vl[3] = {0, 0, 0}, vr[3] = {0, 0, 0};
  if (live) {
    coords3(i, L.nx, L.ny, L.n, c[0], c[1], c[2]);
    dinv = L.w[4 * n + i];
    wd = L.w[3 * n + i];
    ri = L.r[i];
    for (int a = 0; a < 3; ++a) {
      wl[a] = L.w[a * n + i];
      hl[a] = wl[a] != 0 && c[a] > 0;
      if (c[a] + 1 < dim[a]) {
        wr[a] = L.w[a * n + i + stride[a]];
        hr[a] = wr[a] != 0;
      }
    }
    if (WITH_COARSE) {
      vc = ein[i];
      for (int a = 0; a < 3; ++a) {
        if (hl[a]) vl[a] = ein[i - stride[a]];
        if (hr[a]) vr[a] = ein[i + stride[a]];
      }
    }
  }
  pdl_entry();
  if (!live || solve_done(done)) return;
  if (dinv == 0) {
    eout[i] = (T)0;
    return;
  }
  // e plus the coarse correction at the cell and its coupled neighbours
  auto cc = [&](int xx, int yy, int zz) -> T { return C.e[C.at(xx >> 1, yy >> 1, zz >> 1)]; };
  if (WITH_COARSE) {
    vc += cc(c[0], c[1], c[2]);
    for (int a = 0; a < 3; ++a) {
      int p[3] = {c[0], c[1], c[2]};
      if (hl[a]) {
        p[a] = c[a] - 1;
        vl[a] += cc(p[0], p[1], p[2]);
      }
      p[a] = c[a] + 1;
      if (hr[a]) vr[a] += cc(p[0], p[1], p[2]);
    }
  } else {
    vc = ein[i];
    for (int a = 0; a < 3; ++a) {
      if (hl[a]) vl[a] = ein[i - stride[a]];
      if (hr[a]) vr[a] = ein[i + stride[a]];
    }
  }
  T s = wd * vc;
  for (int a = 0; a < 3; ++a) {
    if (hl[a]) s -= wl[a] * vl[a];
    if (hr[a]) s -= wr[a] * vr[a];
  }
  eout[i] = vc + (WITH_COARSE ? L.w1 : L.w2) * dinv * (ri - s);
}

// ------------------------------------------- coarse V-cycle in one block
// Levels lo..hi-1 of the dense hierarchy, staged in shared memory when they
// fit (else worked on in global memory); __syncthreads separates the sweeps.
template <class T>
struct DenseSet {
  DView<T> L[kMaxDense];
  int lo, hi;
};

// One Jacobi sweep of a block-solved level (first: from zero). ce (the next
// coarser level's correction, on a cnx x cny grid) is added to every e first
// when given.
template <class T>
__device__ void blk_jacobi(const DView<T>& L, const T* ein, T* eout, const T* ce, int cnx, int cny, bool first,
                           T om) {
  const int n = (int)L.n;  // block-solved levels hold a few thousand cells: 32-bit index math
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const T* __restrict__ w = L.w;
  const T* __restrict__ r = L.r;
  const float rnx = 1.0f / (float)nx, rny = 1.0f / (float)ny;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const T dinv = w[4 * n + i];
    if (dinv == 0) {
      eout[i] = (T)0;
      continue;
    }
    if (first) {
      eout[i] = om * dinv * r[i];
      continue;
    }
    const int xy = qdiv(i, nx, rnx);
    const int x = i - xy * nx, z = qdiv(xy, ny, rny), y = xy - z * ny;
    auto ev = [&](int j, int xx, int yy, int zz) -> T {
      T v = ein[j];
      if (ce) v += ce[(xx >> 1) + cnx * ((yy >> 1) + cny * (zz >> 1))];
      return v;
    };
    const int c[3] = {x, y, z};
    const int dim[3] = {nx, ny, nz};
    const int stride[3] = {1, nx, nx * ny};
    const T ec = ev(i, x, y, z);
    T s = w[3 * n + i] * ec;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int p[3] = {x, y, z};
      const T wl = w[a * n + i];
      if (wl != 0 && c[a] > 0) {
        p[a] = c[a] - 1;
        s -= wl * ev(i - stride[a], p[0], p[1], p[2]);
      }
      if (c[a] + 1 < dim[a]) {
        const T wr = w[a * n + i + stride[a]];
        if (wr != 0) {
          p[a] = c[a] + 1;
          s -= wr * ev(i + stride[a], p[0], p[1], p[2]);
        }
      }
    }
    eout[i] = ec + om * dinv * (r[i] - s);
  }
}

// Residual of F (correction fe) restricted into C.r.
template <class T>
__device__ void blk_restrict(const DView<T>& F, const T* fe, const DView<T>& C) {
  // one thread per (coarse cell, child), the 8 children on adjacent lanes; the
  // loop runs a whole number of warps so every lane reaches the shuffles
  const int total = ((int)C.n * 8 + 31) & ~31;
  for (int g = threadIdx.x; g < total; g += blockDim.x) {
    const int I = g >> 3, k = g & 7;
    T s = 0;
    if (I < (int)C.n) {
      int X, Y, Z;
      coords3(I, C.nx, C.ny, C.n, X, Y, Z);
      const int x = 2 * X + (k & 1), y = 2 * Y + ((k >> 1) & 1), z = 2 * Z + (k >> 2);
      if (x < F.nx && y < F.ny && z < F.nz) {
        const int i = x + F.nx * (y + F.ny * z);
        if (F.w[4 * F.n + i] != 0) s = F.r[i] - dense_apply(F, fe, i, x, y, z, fe[i]);
      }
    }
    s = sum8(s);
    if (I < (int)C.n && k == 0) C.r[I] = (T)s;
  }
}

// Inverse of the coarsest level's operator (n <= 64 cells), by Gauss-Jordan
// elimination without pivoting (the operator is symmetric positive definite
// once a cell without a stencil is given a unit row). ok = 0 when a pivot is
// not positive (no Dirichlet cell anywhere: the V-cycle then keeps Jacobi sweeps).
template <class T>
__global__ void __launch_bounds__(1024) kd_coarsest_inverse(DView<T> L, double* inv, int* ok) {
  __shared__ double A[64 * 64];
  __shared__ double colk[64];
  const int n = (int)L.n;
  if (n > 64) {
    if (threadIdx.x == 0) *ok = 0;
    return;
  }
  for (int t = threadIdx.x; t < 64 * 64; t += blockDim.x) A[t] = 0.0;
  __syncthreads();
  if ((int)threadIdx.x < n) {
    const int i = threadIdx.x;
    const int xy = i / L.nx;
    const int c[3] = {i - xy * L.nx, xy % L.ny, xy / L.ny};
    const int dim[3] = {L.nx, L.ny, L.nz};
    const int stride[3] = {1, L.nx, L.nx * L.ny};
    if ((double)L.w[4 * L.n + i] == 0) {
      A[i * 64 + i] = 1.0;
    } else {
      A[i * 64 + i] = (double)L.w[3 * L.n + i];
      for (int a = 0; a < 3; ++a) {
        if (c[a] > 0) {
          const int j = i - stride[a];
          if ((double)L.w[4 * L.n + j] != 0) A[i * 64 + j] = -(double)L.w[a * L.n + i];
        }
        if (c[a] + 1 < dim[a]) {
          const int j = i + stride[a];
          if ((double)L.w[4 * L.n + j] != 0) A[i * 64 + j] = -(double)L.w[a * L.n + j];
        }
      }
    }
  }
  for (int k = 0; k < n; ++k) {
    __syncthreads();
    const double p = A[k * 64 + k];
    if (!(p > 1e-300)) {
      if (threadIdx.x == 0) *ok = 0;
      return;
    }
    if ((int)threadIdx.x < n) colk[threadIdx.x] = A[threadIdx.x * 64 + k];
    __syncthreads();
    if ((int)threadIdx.x < n) {
      const int j = threadIdx.x;
      A[k * 64 + j] = (j == k ? 1.0 : A[k * 64 + j]) / p;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
      const int i = t / n, j = t - i * n;
      if (i == k) continue;
      A[i * 64 + j] = (j == k ? 0.0 : A[i * 64 + j]) - colk[i] * A[k * 64 + j];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 64 * 64; t += blockDim.x) inv[t] = A[t];
  if (threadIdx.x == 0) *ok = 1;
}

// Block-wide copy with eight independent loads per thread in flight before
// their stores (one block moves the coarse levels' weights, ~100 KB, into
// shared memory every V-cycle: a load-store chain per element would pay the
// memory latency once per element).
template <class T>
__device__ void blk_copy(T* dst, const T* src, int64_t n) {
  constexpr int U = 8;
  const int64_t step = blockDim.x;
  int64_t i = threadIdx.x;
  for (; i + (U - 1) * step < n; i += U * step) {
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = src[i + u * step];
#pragma unroll
    for (int u = 0; u < U; ++u) dst[i + u * step] = v[u];
  }
  for (; i < n; i += step) dst[i] = src[i];
}

template <class T>
__global__ void __launch_bounds__(1024) kd_coarse_block(DenseSet<T> G, int use_smem, const double* __restrict__ inv,
                                                        const int* __restrict__ inv_ok,
                                                        const int32_t* __restrict__ done) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // Level descriptors live in shared memory (one copy per block); which of a
  // level's two correction buffers is current is a bit in a register.
  __shared__ DView<T> SL[kMaxDense];
  const int lo = G.lo, hi = G.hi;
  if (threadIdx.x == 0) {
    T* p = (T*)smem_raw;
    for (int l = lo; l < hi; ++l) {
      SL[l] = G.L[l];
      if (use_smem) {
        const int64_t n = G.L[l].n;
        SL[l].e = p;
        SL[l].e2 = p + n;
        SL[l].r = p + 2 * n;
        SL[l].w = p + 3 * n;
        p += 9 * n;
      }
    }
  }
  __syncthreads();
  // prologue: the levels' weights (static since the set-up) into shared
  // memory and this thread's entries of the coarsest inverse, while the
  // previous kernel still runs; the residual of level lo is that kernel's
  // output and is copied after the wait
  if (use_smem) {
    for (int l = lo; l < hi; ++l) blk_copy(SL[l].w, G.L[l].w, 6 * SL[l].n);
  }
  const bool exact = *inv_ok && SL[hi - 1].n <= 64;
  double iv[4] = {0.0, 0.0, 0.0, 0.0};
  if (exact) {
    const int n = (int)SL[hi - 1].n;
    const int i = threadIdx.x >> 4, p = threadIdx.x & 15;
    if (i < n) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = p + 16 * q;
        if (j < n) iv[q] = inv[i * 64 + j];
      }
    }
  }
  pdl_entry();
  if (solve_done(done)) return;
  if (use_smem) {
    blk_copy(SL[lo].r, G.L[lo].r, SL[lo].n);
    __syncthreads();
  }
  unsigned swapped = 0;
  auto cur = [&](int l) -> T* { return ((swapped >> l) & 1) ? SL[l].e2 : SL[l].e; };
  auto oth = [&](int l) -> T* { return ((swapped >> l) & 1) ? SL[l].e : SL[l].e2; };
  // down
  for (int l = lo; l < hi - 1; ++l) {
    const DView<T>& L = SL[l];
    blk_jacobi(L, cur(l), cur(l), (const T*)nullptr, 0, 0, true, L.w1);
    __syncthreads();
    blk_jacobi(L, cur(l), oth(l), (const T*)nullptr, 0, 0, false, L.w2);
    __syncthreads();
    swapped ^= 1u << l;
    blk_restrict(L, cur(l), SL[l + 1]);
    __syncthreads();
  }
  // coarsest: exact solve with the set-up's inverse, else Jacobi sweeps from zero
  {
    const int l = hi - 1;
    const DView<T>& L = SL[l];
    if (exact) {
      // row i of inv r by the 16 lanes i*16..i*16+15 (j = lane part + 16 q),
      // summed over the lanes with shuffles; the block holds 1024 threads
      const int n = (int)L.n;
      const int i = threadIdx.x >> 4, p = threadIdx.x & 15;
      double s = 0.0;
      if (i < n) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int j = p + 16 * q;
          if (j < n) s += iv[q] * (double)L.r[j];
        }
      }
#pragma unroll
      for (int m = 8; m > 0; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m, 16);
      if (i < n && p == 0) cur(l)[i] = (double)L.w[4 * L.n + i] == 0 ? (T)0 : (T)s;
      __syncthreads();
    } else {
      blk_jacobi(L, cur(l), cur(l), (const T*)nullptr, 0, 0, true, L.w1);
      __syncthreads();
      for (int s = 1; s < kCoarsestSweeps; ++s) {
        blk_jacobi(L, cur(l), oth(l), (const T*)nullptr, 0, 0, false, (s & 1) ? L.w2 : L.w1);
        __syncthreads();
        swapped ^= 1u << l;
      }
    }
  }
  // up
  for (int l = hi - 2; l >= lo; --l) {
    const DView<T>& L = SL[l];
    blk_jacobi(L, cur(l), oth(l), cur(l + 1), SL[l + 1].nx, SL[l + 1].ny, false, L.w1);
    __syncthreads();
    blk_jacobi(L, oth(l), cur(l), (const T*)nullptr, 0, 0, false, L.w2);
    __syncthreads();
  }
  if (use_smem || cur(lo) != G.L[lo].e) blk_copy(G.L[lo].e, cur(lo), SL[lo].n);
}

// ------------------------------------------------------------ weights setup
// Level-1 weights from the level-0 face classes (Galerkin, piecewise constant).
template <class T>
__global__ void kw_l1(const int* __restrict__ dbl, int nd, const uint16_t* __restrict__ fmask, T* w, size_t ncap1,
                      Params P, double scale) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nd * 64) return;
  int b = dbl[g >> 6];
  int o = (int)(g & 63);
  int X = o & 3, Y = (o >> 2) & 3, Z = o >> 4;
  double wl[3] = {0, 0, 0}, dd = 0;
  for (int k = 0; k < 8; ++k) {
    int x = 2 * X + (k & 1), y = 2 * Y + ((k >> 1) & 1), z = 2 * Z + (k >> 2);
    uint16_t m = fmask[(size_t)b * kCells + x + 8 * y + 64 * z];
    if (!(m & kDomainBit)) continue;
    for (int f = 0; f < 6; ++f)
      if ((m & (1u << (8 + f))) && !(m & (1u << f))) dd += P.ih2[f >> 1];
    int lc[3] = {k & 1, (k >> 1) & 1, k >> 2};
    for (int a = 0; a < 3; ++a)
      if (lc[a] == 0 && (m & (1u << (2 * a)))) wl[a] += P.ih2[a];
  }
  size_t i = (size_t)b * 64 + o;
  for (int a = 0; a < 3; ++a) w[a * ncap1 + i] = (T)(scale * wl[a]);
  w[5 * ncap1 + i] = (T)(scale * dd);
}

// Brick level D -> D/2 (D = 4), or D = 2 -> dense level 3 at the brick position.
template <class T, int D>
__global__ void kw_coarsen(const int* __restrict__ dbl, int nd, const int* __restrict__ bkey, const T* __restrict__ wf,
                           size_t ncapf, T* wc, size_t ncapc, DenseGrid g3, double scale) {
  constexpr int H = D / 2;
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nd * H * H * H) return;
  int b = dbl[g / (H * H * H)];
  int o = (int)(g % (H * H * H));
  int X = o % H, Y = (o / H) % H, Z = o / (H * H);
  double wl[3] = {0, 0, 0}, dd = 0;
  for (int k = 0; k < 8; ++k) {
    int lc[3] = {k & 1, (k >> 1) & 1, k >> 2};
    size_t fi = (size_t)b * D * D * D + (2 * X + lc[0]) + D * (2 * Y + lc[1]) + D * D * (2 * Z + lc[2]);
    dd += (double)wf[5 * ncapf + fi];
    for (int a = 0; a < 3; ++a)
      if (lc[a] == 0) wl[a] += (double)wf[a * ncapf + fi];
  }
  size_t i = D == 2 ? (size_t)g3.index(bkey[3 * b], bkey[3 * b + 1], bkey[3 * b + 2])
                    : (size_t)b * H * H * H + o;
  for (int a = 0; a < 3; ++a) wc[a * ncapc + i] = (T)(scale * wl[a]);
  wc[5 * ncapc + i] = (T)(scale * dd);
}

template <class T, int D>
__global__ void kw_diag(const int* __restrict__ dbl, int nd, const int* __restrict__ nbr, T* w, size_t ncap) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nd * D * D * D) return;
  int b = dbl[g / (D * D * D)];
  int o = (int)(g % (D * D * D));
  int x = o % D, y = (o / D) % D, z = o / (D * D);
  size_t i = (size_t)b * D * D * D + o;
  double d = (double)w[5 * ncap + i];
  for (int a = 0; a < 3; ++a) {
    d += (double)w[a * ncap + i];
    int p[3] = {x, y, z};
    p[a] += 1;
    int64_t n = lidx<D>(nbr, b, p[0], p[1], p[2]);
    if (n >= 0) d += (double)w[a * ncap + n];
  }
  w[3 * ncap + i] = (T)d;
  w[4 * ncap + i] = d > 0 ? (T)(1.0 / d) : (T)0;
}

template <class T>
__global__ void kwd_coarsen(DView<T> F, DView<T> C, double scale) {
  int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= C.n) return;
  int X = (int)(I % C.nx), Y = (int)((I / C.nx) % C.ny), Z = (int)(I / ((int64_t)C.nx * C.ny));
  double wl[3] = {0, 0, 0}, dd = 0;
  for (int k = 0; k < 8; ++k) {
    int lc[3] = {k & 1, (k >> 1) & 1, k >> 2};
    int x = 2 * X + lc[0], y = 2 * Y + lc[1], z = 2 * Z + lc[2];
    if (x >= F.nx || y >= F.ny || z >= F.nz) continue;
    int64_t i = F.at(x, y, z);
    dd += (double)F.w[5 * F.n + i];
    for (int a = 0; a < 3; ++a)
      if (lc[a] == 0) wl[a] += (double)F.w[a * F.n + i];
  }
  for (int a = 0; a < 3; ++a) C.w[a * C.n + I] = (T)(scale * wl[a]);
  C.w[5 * C.n + I] = (T)(scale * dd);
}

template <class T>
__global__ void kwd_diag(DView<T> L) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  int x = (int)(i % L.nx), y = (int)((i / L.nx) % L.ny), z = (int)(i / ((int64_t)L.nx * L.ny));
  int c[3] = {x, y, z};
  int dim[3] = {L.nx, L.ny, L.nz};
  int64_t stride[3] = {1, L.nx, (int64_t)L.nx * L.ny};
  double d = (double)L.w[5 * L.n + i];
  for (int a = 0; a < 3; ++a) {
    d += (double)L.w[a * L.n + i];
    if (c[a] + 1 < dim[a]) d += (double)L.w[a * L.n + i + stride[a]];
  }
  L.w[3 * L.n + i] = (T)d;
  L.w[4 * L.n + i] = d > 0 ? (T)(1.0 / d) : (T)0;
}

// ------------------------------------------------------------ host side
template <class T>
static DView<T> dview(Ctx* c, int l) {
  DView<T> v;
  const DenseDesc& d = c->dense[l];
  v.nx = d.nx;
  v.ny = d.ny;
  v.nz = d.nz;
  v.n = d.n;
  T* base = (T*)c->dense_buf;
  v.e = base + 9 * d.off;
  v.e2 = v.e + d.n;
  v.r = v.e + 2 * d.n;
  v.w = v.e + 3 * d.n;
  v.w1 = (T)c->dp.mgw1;
  v.w2 = (T)c->dp.mgw2;
  return v;
}

// Lays out the dense levels for the current bounding box (level 3 = one cell
// per brick) and grows the buffer when needed.
static int dense_layout(Ctx* c) {
  int* bb = c->hs->bbox;
  int nx = bb[3] - bb[0] + 1, ny = bb[4] - bb[1] + 1, nz = bb[5] - bb[2] + 1;
  if (nx < 1 || ny < 1 || nz < 1) nx = ny = nz = 1;
  c->g3.x0 = bb[0];
  c->g3.y0 = bb[1];
  c->g3.z0 = bb[2];
  c->g3.nx = nx;
  c->g3.ny = ny;
  c->g3.nz = nz;
  int nl = 0;
  int64_t off = 0;
  while (nl < kMaxDense) {
    DenseDesc& d = c->dense[nl];
    d.nx = nx;
    d.ny = ny;
    d.nz = nz;
    d.n = (int64_t)nx * ny * nz;
    d.off = off;
    off += d.n;
    ++nl;
    if (d.n <= 64 || (nx <= 2 && ny <= 2 && nz <= 2)) break;
    nx = (nx + 1) / 2;
    ny = (ny + 1) / 2;
    nz = (nz + 1) / 2;
  }
  c->ndense = nl;
  size_t ts = c->mg_float ? 4 : 8;
  size_t need = (size_t)off * 9 * ts;
  if (need > c->dense_bytes) {
    cudaFree(c->dense_buf);
    c->dense_buf = nullptr;
    c->dense_bytes = 0;
    int rc = check(cudaMalloc(&c->dense_buf, need + need / 4));
    if (rc) return rc;
    c->dense_bytes = need + need / 4;
  }
  // levels above blk_max_cells run as device-wide sweeps (level 3 always);
  // the rest go to the one-block solve, staged in shared memory (9 arrays per
  // cell) when they fit
  int lo = 1;
  while (lo < nl - 1 && c->dense[lo].n > c->blk_max_cells) ++lo;
  c->dense_lo = lo;
  int64_t cells = 0;
  for (int l = lo; l < nl; ++l) cells += c->dense[l].n;
  c->dense_smem = (size_t)cells * 9 * ts;
  return check(cudaMemsetAsync(c->dense_buf, 0, (size_t)off * 9 * ts, c->stream));
}

template <class T>
static int mg_setup_t(Ctx* c) {
  cudaStream_t st = c->stream;
  int nd = c->ndom_host;
  int rc = dense_layout(c);
  if (rc) return rc;
  size_t ncap1 = (size_t)c->cap_bricks * 64, ncap2 = (size_t)c->cap_bricks * 8;
  T* w1 = (T*)c->mg_w[1];
  T* w2 = (T*)c->mg_w[2];
  DView<T> d3 = dview<T>(c, 0);
  int g1 = grid_for((int64_t)nd * 64, 256), g2 = grid_for((int64_t)nd * 8, 256), g3 = grid_for(nd, 256);
  // Bricks without a domain cell keep zero weights, so stencils never couple to them.
  rc = check(cudaMemsetAsync(w1, 0, ncap1 * 6 * sizeof(T), st));
  if (!rc) rc = check(cudaMemsetAsync(w2, 0, ncap2 * 6 * sizeof(T), st));
  if (rc) return rc;
  const double sc = c->mg_scale;
  kw_l1<T><<<g1, 256, 0, st>>>(c->dbl, nd, c->fmask, w1, ncap1, c->dp, sc); MAC_COUNT(c);
  kw_coarsen<T, 4><<<g2, 256, 0, st>>>(c->dbl, nd, c->bkey, w1, ncap1, w2, ncap2, c->g3, sc); MAC_COUNT(c);
  kw_coarsen<T, 2><<<g3, 256, 0, st>>>(c->dbl, nd, c->bkey, w2, ncap2, d3.w, (size_t)d3.n, c->g3, sc); MAC_COUNT(c);
  for (int l = 0; l + 1 < c->ndense; ++l) {
    DView<T> F = dview<T>(c, l), C = dview<T>(c, l + 1);
    kwd_coarsen<T><<<grid_for(C.n, 256), 256, 0, st>>>(F, C, sc); MAC_COUNT(c);
  }
  kw_diag<T, 4><<<g1, 256, 0, st>>>(c->dbl, nd, c->nbr, w1, ncap1); MAC_COUNT(c);
  kw_diag<T, 2><<<g2, 256, 0, st>>>(c->dbl, nd, c->nbr, w2, ncap2); MAC_COUNT(c);
  for (int l = 0; l < c->ndense; ++l) {
    DView<T> L = dview<T>(c, l);
    kwd_diag<T><<<grid_for(L.n, 256), 256, 0, st>>>(L); MAC_COUNT(c);
  }
  kd_coarsest_inverse<T><<<1, 1024, 0, st>>>(dview<T>(c, c->ndense - 1), c->coarse_inv, c->coarse_ok); MAC_COUNT(c);
  return check(cudaGetLastError());
}

int mg_setup(Ctx* c) { return c->mg_float ? mg_setup_t<float>(c) : mg_setup_t<double>(c); }

// part: 1 = the head (first kernel, with update the convergence test), 2 = the rest.
template <class T>
static void mg_vcycle_t(Ctx* c, int update, int part) {
  int nd = c->ndom_host;
  size_t ncap1 = (size_t)c->cap_bricks * 64, ncap2 = (size_t)c->cap_bricks * 8;
  T* e0 = (T*)c->mg_e[0];
  T* e0b = (T*)c->mg_e2[0];
  T* e1 = (T*)c->mg_e[1];
  T* e1b = (T*)c->mg_e2[1];
  T* e2 = (T*)c->mg_e[2];
  T* e2b = (T*)c->mg_e2[2];
  T* r1 = (T*)c->mg_r[1];
  T* r2 = (T*)c->mg_r[2];
  T* w1 = (T*)c->mg_w[1];
  T* w2 = (T*)c->mg_w[2];
  DView<T> d3 = dview<T>(c, 0);
  int g1 = grid_for((int64_t)nd * 64, 256), g2 = grid_for((int64_t)nd * 8, 256);
  DenseGrid G = c->g3;
  const int32_t* dn = &c->ds->done;
  // down (with update: finish the previous CG iteration into r2, which becomes r)
  const bool one = c->mg_sweeps0 == 1;
  if (part & 1) {
    c->npart_head = nd;
    if (c->mg_bulk && c->bulk_grid > 0) {
      const int g = nd < c->bulk_grid ? nd : c->bulk_grid;
      c->npart_head = g;
      if (one)
        launch_k(c, k0_head_bulk<T, true>, g, kBT, bulk_smem<T>(), c->dbl, nd, c->nbr, c->fmask, c->r, c->r2, c->x, c->pd,
                 c->q, c->partial, c->ds, update, e0, r1, c->dp);
      else
        launch_k(c, k0_head_bulk<T, false>, g, kBT, bulk_smem<T>(), c->dbl, nd, c->nbr, c->fmask, c->r, c->r2, c->x,
                 c->pd, c->q, c->partial, c->ds, update, e0, r1, c->dp);
      MAC_COUNT(c);
    } else if (one) {
      launch_k(c, k0_pre_restrict<T>, nd, kBT, 0, c->drow, c->fmask, c->r, c->r2, c->x, c->pd, c->q, c->partial,
               c->ds, update, r1, c->dp); MAC_COUNT(c);
    } else {
      launch_k(c, k0_pre<T>, nd, kBT, 0, c->drow, c->fmask, c->r, c->r2, c->x, c->pd, c->q, c->partial, c->ds,
               update, e0, c->dp); MAC_COUNT(c);
    }
    if (update) {
      std::swap(c->r, c->r2);
      cg_finish_update(c);
    }
  }
  if (!(part & 2)) return;
  if (!one) {
    launch_k(c, k0_restrict<T>, nd, kBT, 0, c->drow, c->fmask, c->r, e0, r1, c->dp, dn); MAC_COUNT(c);
  }
  const T sw1 = (T)c->dp.mgw1, sw2 = (T)c->dp.mgw2;
  launch_k(c, kl_pre<T, 4>, g1, 256, 0, c->drow, nd, w1, ncap1, r1, e1, sw1, sw2, dn); MAC_COUNT(c);
  launch_k(c, kl_restrict<T, 4>, g1, 256, 0, c->drow, nd, c->bkey, w1, ncap1, r1, e1, r2, G, dn); MAC_COUNT(c);
  launch_k(c, kl_pre<T, 2>, g2, 256, 0, c->drow, nd, w2, ncap2, r2, e2, sw1, sw2, dn); MAC_COUNT(c);
  launch_k(c, kl_restrict<T, 2>, g2, 256, 0, c->drow, nd, c->bkey, w2, ncap2, r2, e2, d3.r, G, dn); MAC_COUNT(c);
  // dense level 3 on the device, levels 4.. in one block
  if (c->ndense > 1) {
    // dense levels 0 .. lo-1 device-wide, lo .. in one block
    const int lo = c->dense_lo;
    for (int l = 0; l < lo; ++l) {
      const DView<T> L = dview<T>(c, l), C = dview<T>(c, l + 1);
      launch_k(c, kd_pre<T>, grid_for(L.n, 256), 256, 0, L, dn); MAC_COUNT(c);
      launch_k(c, kd_restrict<T>, grid_for(8 * C.n, 256), 256, 0, L, C, dn); MAC_COUNT(c);
    }
    DenseSet<T> S;
    for (int l = 0; l < c->ndense; ++l) S.L[l] = dview<T>(c, l);
    S.lo = lo;
    S.hi = c->ndense;
    int use_smem = c->dense_smem <= (size_t)c->smem_optin ? 1 : 0;
    launch_k(c, kd_coarse_block<T>, 1, 1024, use_smem ? c->dense_smem : 0, S, use_smem, c->coarse_inv, c->coarse_ok,
             dn); MAC_COUNT(c);
    for (int l = lo - 1; l >= 0; --l) {
      const DView<T> L = dview<T>(c, l), C = dview<T>(c, l + 1);
      launch_k(c, kd_jacobi<T, true>, grid_for(L.n, 256), 256, 0, L, L.e, L.e2, C, dn); MAC_COUNT(c);
      launch_k(c, kd_jacobi<T, false>, grid_for(L.n, 256), 256, 0, L, L.e2, L.e, C, dn); MAC_COUNT(c);
    }
  } else {
    DenseSet<T> S;
    S.L[0] = d3;
    S.lo = 0;
    S.hi = 1;
    launch_k(c, kd_coarse_block<T>, 1, 1024, 0, S, 0, c->coarse_inv, c->coarse_ok, dn); MAC_COUNT(c);
  }
  // up
  launch_k(c, kl_jacobi<T, 2, true>, g2, 256, 0, c->drow, nd, c->bkey, w2, ncap2, r2, e2, d3.e, e2b, G, sw1,
           dn); MAC_COUNT(c);
  launch_k(c, kl_jacobi<T, 2, false>, g2, 256, 0, c->drow, nd, c->bkey, w2, ncap2, r2, e2b, nullptr, e2, G,
           sw2, dn); MAC_COUNT(c);
  launch_k(c, kl_jacobi<T, 4, true>, g1, 256, 0, c->drow, nd, c->bkey, w1, ncap1, r1, e1, e2, e1b, G, sw1,
           dn); MAC_COUNT(c);
  launch_k(c, kl_jacobi<T, 4, false>, g1, 256, 0, c->drow, nd, c->bkey, w1, ncap1, r1, e1b, nullptr, e1, G,
           sw2, dn); MAC_COUNT(c);
  if (one) {
    launch_k(c, k0_post_one<T>, nd, kBT, 0, c->drow, c->fmask, c->r, e1, c->z, c->partial, c->dp, dn); MAC_COUNT(c);
    return;
  }
  launch_k(c, k0_post<T, true>, nd, kBT, 0, c->drow, c->fmask, c->r, e0, e1, e0b, nullptr, nullptr, c->dp,
           dn); MAC_COUNT(c);
  launch_k(c, k0_post<T, false>, nd, kBT, 0, c->drow, c->fmask, c->r, e0b, nullptr, nullptr, c->z, c->partial,
           c->dp, dn); MAC_COUNT(c);
}

void mg_vcycle(Ctx* c, int update, int part) {
  if (c->mg_float) mg_vcycle_t<float>(c, update, part);
  else mg_vcycle_t<double>(c, update, part);
}

int mg_configure(Ctx* c) {
  int dev = c->prm.device, optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  // the dynamic part may use what the kernel's static shared memory leaves
  cudaFuncAttributes fa64, fa32;
  int rc = check(cudaFuncGetAttributes(&fa64, kd_coarse_block<double>));
  if (!rc) rc = check(cudaFuncGetAttributes(&fa32, kd_coarse_block<float>));
  if (rc) return rc;
  const int dyn64 = optin - (int)fa64.sharedSizeBytes, dyn32 = optin - (int)fa32.sharedSizeBytes;
  c->smem_optin = dyn64 < dyn32 ? dyn64 : dyn32;
  rc = check(cudaFuncSetAttribute(kd_coarse_block<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn64));
  if (!rc) rc = check(cudaFuncSetAttribute(kd_coarse_block<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn32));
  // the prefetching first kernel: as many blocks as fit on all SMs at once
  int nsm = 0, occ = 0;
  if (!rc) rc = check(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (c->mg_float) {
    if (!rc) rc = check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k0_head_bulk<float, true>, kBT,
                                                                      bulk_smem<float>()));
  } else {
    if (!rc) rc = check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k0_head_bulk<double, true>, kBT,
                                                                      bulk_smem<double>()));
  }
  c->bulk_grid = rc ? 0 : nsm * occ;
  return rc;
}

}  // namespace mac

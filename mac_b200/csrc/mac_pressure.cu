// Pressure projection on the brick grid: Algorithms_Solve_Pressure
// (src/Algorithms_Solve_Pressure.h:44-222) with Policy_Divergence,
// Policy_Gradiant, Policy_Von_Neumann_Boundary and Policy_Pressure_If_Correction,
// solving the same ghost-fluid system the reference assembles for Umfpack, but
// matrix-free and iteratively:
//
//   A p = div u,  A = 7-point Laplacian over in-domain cells; per face of an
//   in-domain cell c: missing neighbour or non-domain neighbour -> Dirichlet
//   (p = 0, diagonal only); const face -> Neumann (nothing); in-domain
//   neighbour -> coupling 1/h^2.
//
// We solve M x = -div u with M = -A (symmetric positive definite) by CG in
// FP64, preconditioned by a multigrid V-cycle on brick-local levels
// (8^3, 4^3, 2^3, 1 cell per brick). Coarse operators are the Galerkin
// products with piecewise-constant transfer, scaled by 1/2 per level; they are
// stored as left-face weights plus a Dirichlet diagonal. The V-cycle runs in
// FP64 (plain form) or FP32 (mixed form); the CG recurrences, dot products and
// the final divergence check are always FP64.
#include <cstdio>
#include <cstring>

#include "mac_internal.cuh"

namespace mac {

constexpr int kVecBlocks = 148 * 8;  // fixed grid for reductions (deterministic order)
constexpr double kOmega = 0.8;
constexpr double kCoarseScale = 0.5;
constexpr int kCoarseSweeps = 24;

// face bit f = 2*axis + (sign > 0)
constexpr uint16_t kDomainBit = 0x8000;

// ------------------------------------------------------------ allocation
template <class T>
static int dalloc(T** p, size_t n) {
  return check(cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)));
}

int alloc_solver(Ctx* c) {
  size_t nc = (size_t)c->cap_bricks * kCells;
  int rc = MAC_OK;
  auto A = [&](int r) { if (rc == MAC_OK) rc = r; };
  A(dalloc(&c->fmask, nc));
  A(dalloc(&c->x, nc));
  A(dalloc(&c->b, nc));
  A(dalloc(&c->r, nc));
  A(dalloc(&c->z, nc));
  A(dalloc(&c->pd, nc));
  A(dalloc(&c->q, nc));
  c->npartial = kVecBlocks * 2;
  A(dalloc(&c->partial, c->npartial));
  c->mg_float = c->prm.solver == MAC_SOLVER_MGPCG_MIXED;
  size_t ts = c->mg_float ? 4 : 8;
  for (int l = 0; l < kLevels; ++l) {
    size_t n = (size_t)c->cap_bricks * (size_t)((8 >> l) * (8 >> l) * (8 >> l));
    A(check(cudaMalloc(&c->mg_e[l], ts * n)));
    A(check(cudaMalloc(&c->mg_e2[l], ts * n)));
    if (l > 0) {
      A(check(cudaMalloc(&c->mg_r[l], ts * n)));
      A(check(cudaMalloc(&c->mg_w[l], ts * n * 6)));
    }
  }
  if (rc == MAC_OK) {
    cudaMemset(c->x, 0, 8 * nc);
    cudaMemset(c->fmask, 0, 2 * nc);
  }
  return rc;
}

void free_solver(Ctx* c) {
  cudaFree(c->fmask); cudaFree(c->x); cudaFree(c->b); cudaFree(c->r); cudaFree(c->z); cudaFree(c->pd);
  cudaFree(c->q); cudaFree(c->partial);
  for (int l = 0; l < kLevels; ++l) {
    cudaFree(c->mg_e[l]); cudaFree(c->mg_e2[l]); cudaFree(c->mg_r[l]); cudaFree(c->mg_w[l]);
  }
}

// ------------------------------------------------------------ helpers
template <int D>
__device__ inline int64_t lidx(const int* __restrict__ nbr, int b, int x, int y, int z) {
  int dx = x < 0 ? -1 : (x >= D ? 1 : 0);
  int dy = y < 0 ? -1 : (y >= D ? 1 : 0);
  int dz = z < 0 ? -1 : (z >= D ? 1 : 0);
  int nb = ((dx | dy | dz) == 0) ? b : nbr[(size_t)b * kNbr + nbr_index(dx, dy, dz)];
  if (nb < 0) return -1;
  return (int64_t)nb * (D * D * D) + (x - D * dx) + D * (y - D * dy) + D * D * (z - D * dz);
}

__device__ inline bool in_domain(const int8_t* __restrict__ lay, const uint8_t* __restrict__ type, int64_t i) {
  return i >= 0 && lay[i] != kMissing && is_fluid(type[i]);
}

// Block reduction of up to 2 doubles into partial[blockIdx.x] / partial[gridDim.x + blockIdx.x].
__device__ inline void block_reduce2(double a, double b, double* partial) {
  __shared__ double sa[32], sb[32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (w == 0) {
    int nw = blockDim.x >> 5;
    a = l < nw ? sa[l] : 0.0;
    b = l < nw ? sb[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (l == 0) {
      partial[blockIdx.x] = a;
      partial[gridDim.x + blockIdx.x] = b;
    }
  }
}

// Sums the partials in a fixed order (one block).
__device__ inline void sum_partials(const double* partial, int nblk, double* s0, double* s1) {
  __shared__ double sa[32], sb[32];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    a += partial[i];
    b += partial[nblk + i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      ta += sa[i];
      tb += sb[i];
    }
    *s0 = ta;
    *s1 = tb;
  }
}

// ------------------------------------------------------- system set-up
// Face classes of every in-domain cell (the assembly loop of
// src/Algorithms_Solve_Pressure.h:103-136): bit f (interior coupling) and bit
// 8+f (face counts in the diagonal); Neumann faces have neither. The Neumann
// test is Data_CellType_Interface_Constant::GetIsConstantInterface_Impl
// (src/Data_CellType_Interface_Constant.h:45-61): only for a valid neighbour;
// sign +1 looks at the neighbour's left face, sign -1 at the cell's own.
__global__ void k_fmask(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                        const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                        const uint8_t* __restrict__ flags, uint16_t* fmask, Scalars* ds) {
  int cnt = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    uint16_t m = 0;
    if (lay[c] != kMissing && is_fluid(type[c])) {
      ++cnt;
      m = kDomainBit;
      int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
      for (int f = 0; f < 6; ++f) {
        int ax = f >> 1, s = (f & 1) ? 1 : -1;
        int p[3] = {x, y, z};
        p[ax] += s;
        int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
        if (n < 0 || lay[n] == kMissing) {
          m |= (uint16_t)(1u << (8 + f));  // missing neighbour: Dirichlet
          continue;
        }
        bool neumann = s > 0 ? ((flags[n] >> ax) & 1) : ((flags[c] >> ax) & 1);
        if (neumann) continue;
        m |= (uint16_t)(1u << (8 + f));
        if (is_fluid(type[n])) m |= (uint16_t)(1u << f);
      }
    }
    fmask[c] = m;
  }
  __shared__ int sc;
  if (threadIdx.x == 0) sc = 0;
  __syncthreads();
  atomicAdd(&sc, cnt);
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd((unsigned long long*)&ds->nunknown, (unsigned long long)sc);
}

__global__ void k_zero_unknown(Scalars* ds) { ds->nunknown = 0; }

__device__ inline double diag0(uint16_t m, const Params& P) {
  double d = 0;
  for (int f = 0; f < 6; ++f)
    if (m & (1u << (8 + f))) d += P.ih2[f >> 1];
  return d;
}

// Level-1 weights from the level-0 face classes. w layout (per level, 6
// slots of ncap entries): [0..2] left-face weights x,y,z, [3] diagonal,
// [4] inverse diagonal (0 outside the domain), [5] Dirichlet part of the
// diagonal. Galerkin product with piecewise-constant transfer: a coarse face
// weight is the sum of the interior fine faces across it, the Dirichlet part
// the sum of the children's; faces between two in-domain siblings cancel.
// Every level is scaled by kCoarseScale.
template <class T>
__global__ void k_weights_l1(const int* __restrict__ blist, int nlive, const uint16_t* __restrict__ fmask, T* w,
                             size_t ncap1, Params P) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * 64;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 6];
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
    for (int a = 0; a < 3; ++a) w[a * ncap1 + i] = (T)(kCoarseScale * wl[a]);
    w[5 * ncap1 + i] = (T)(kCoarseScale * dd);
  }
}

// Level with edge D/2 from level with edge D.
template <class T, int D>
__global__ void k_weights_coarsen(const int* __restrict__ blist, int nlive, const T* __restrict__ wf, size_t ncapf,
                                  T* wc, size_t ncapc) {
  constexpr int H = D / 2;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * H * H * H;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g / (H * H * H)];
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
    size_t i = (size_t)b * H * H * H + o;
    for (int a = 0; a < 3; ++a) wc[a * ncapc + i] = (T)(kCoarseScale * wl[a]);
    wc[5 * ncapc + i] = (T)(kCoarseScale * dd);
  }
}

// Diagonal = Dirichlet part + the six face weights (own left faces and the
// right neighbours' left faces); inverse 0 for cells with no domain child.
template <class T, int D>
__global__ void k_weights_diag(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr, T* w,
                               size_t ncap) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * D * D * D;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g / (D * D * D)];
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
}

// ------------------------------------------------------------ operators
// Level 0: M e(c) = diag(c) e(c) - sum over interior faces ih2 * e(n).
template <class TV>
struct L0 {
  __device__ static inline double apply(const TV* __restrict__ e, const int* __restrict__ nbr, int b, int x, int y,
                                        int z, uint16_t m, double ec, const Params& P) {
    double s = diag0(m, P) * ec;
    for (int f = 0; f < 6; ++f) {
      if (!(m & (1u << f))) continue;
      int p[3] = {x, y, z};
      p[f >> 1] += (f & 1) ? 1 : -1;
      int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
      s -= P.ih2[f >> 1] * (double)e[n];
    }
    return s;
  }
};

// Levels >= 1 (edge D): M e(C) = diag e(C) - sum_a [wl_a(C) e(C-e_a) + wl_a(C+e_a) e(C+e_a)].
template <class T, int D>
__device__ inline double apply_l(const T* __restrict__ e, const T* __restrict__ w, size_t ncap,
                                 const int* __restrict__ nbr, int b, int x, int y, int z, size_t i, double ec) {
  double s = (double)w[3 * ncap + i] * ec;
  for (int a = 0; a < 3; ++a) {
    double wl = (double)w[a * ncap + i];
    if (wl != 0) {
      int p[3] = {x, y, z};
      p[a] -= 1;
      int64_t n = lidx<D>(nbr, b, p[0], p[1], p[2]);
      if (n >= 0) s -= wl * (double)e[n];
    }
    int p[3] = {x, y, z};
    p[a] += 1;
    int64_t n = lidx<D>(nbr, b, p[0], p[1], p[2]);
    if (n >= 0) {
      double wr = (double)w[a * ncap + n];
      if (wr != 0) s -= wr * (double)e[n];
    }
  }
  return s;
}

// ---------------------------------------------------------- V-cycle: level 0
// Two Jacobi sweeps from zero, fused: e1 = w Dinv r; e = e1 + w Dinv (r - M e1).
template <class T>
__global__ void __launch_bounds__(256) k_pre0(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                              const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                              T* __restrict__ e, Params P) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    uint16_t m = fmask[c];
    if (!(m & kDomainBit)) {
      e[c] = (T)0;
      continue;
    }
    double dc = diag0(m, P);
    double dinv = dc > 0 ? 1.0 / dc : 0.0;
    double rc = r[c];
    double e1c = kOmega * dinv * rc;
    int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
    double s = dc * e1c;
    for (int f = 0; f < 6; ++f) {
      if (!(m & (1u << f))) continue;
      int p[3] = {x, y, z};
      p[f >> 1] += (f & 1) ? 1 : -1;
      int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
      double dn = diag0(fmask[n], P);
      double e1n = dn > 0 ? kOmega * (1.0 / dn) * r[n] : 0.0;
      s -= P.ih2[f >> 1] * e1n;
    }
    e[c] = (T)(e1c + kOmega * dinv * (rc - s));
  }
}

// Residual of level 0 restricted to level 1: rc(C) = sum over 8 children of (r - M e).
template <class T>
__global__ void __launch_bounds__(256) k_restrict0(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                   const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                                   const T* __restrict__ e, T* __restrict__ rc1, Params P) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * 64;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 6];
    int o = (int)(g & 63);
    int X = o & 3, Y = (o >> 2) & 3, Z = o >> 4;
    double s = 0;
    for (int k = 0; k < 8; ++k) {
      int x = 2 * X + (k & 1), y = 2 * Y + ((k >> 1) & 1), z = 2 * Z + (k >> 2);
      int64_t c = (int64_t)b * kCells + x + 8 * y + 64 * z;
      uint16_t m = fmask[c];
      if (!(m & kDomainBit)) continue;
      s += r[c] - L0<T>::apply(e, nbr, b, x, y, z, m, (double)e[c], P);
    }
    rc1[(size_t)b * 64 + o] = (T)s;
  }
}

// Post-smoothing sweep 1 with the coarse correction added on the fly:
// ep = e + P ec; out = ep + w Dinv (r - M ep). Sweep 2 (POST2) is a plain
// Jacobi sweep writing the FP64 preconditioned residual z and its dot with r.
template <class T, bool WITH_COARSE>
__global__ void __launch_bounds__(256) k_post0(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                               const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                               const T* __restrict__ e, const T* __restrict__ ec1, T* __restrict__ eout,
                                               double* __restrict__ zout, double* partial, Params P) {
  double rz = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    uint16_t m = fmask[c];
    if (!(m & kDomainBit)) {
      if (WITH_COARSE) eout[c] = (T)0;
      else zout[c] = 0.0;
      continue;
    }
    int x = o & 7, y = (o >> 3) & 7, z = o >> 6;
    auto ep = [&](int64_t n, int bx, int xx, int yy, int zz) -> double {
      double v = (double)e[n];
      if (WITH_COARSE) v += (double)ec1[(size_t)bx * 64 + (xx >> 1) + 4 * (yy >> 1) + 16 * (zz >> 1)];
      return v;
    };
    double epc = ep(c, b, x, y, z);
    double dc = diag0(m, P);
    double s = dc * epc;
    for (int f = 0; f < 6; ++f) {
      if (!(m & (1u << f))) continue;
      int p[3] = {x, y, z};
      p[f >> 1] += (f & 1) ? 1 : -1;
      int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
      int nb = (int)(n >> 9);
      int no = (int)(n & 511);
      s -= P.ih2[f >> 1] * ep(n, nb, no & 7, (no >> 3) & 7, no >> 6);
    }
    double dinv = dc > 0 ? 1.0 / dc : 0.0;
    double out = epc + kOmega * dinv * (r[c] - s);
    if (WITH_COARSE) {
      eout[c] = (T)out;
    } else {
      zout[c] = out;
      rz += r[c] * out;
    }
  }
  if (!WITH_COARSE) block_reduce2(rz, 0.0, partial);
}

// ------------------------------------------------------- V-cycle: levels >= 1
template <class T, int D>
__global__ void __launch_bounds__(256) k_pre_l(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                               const T* __restrict__ w, size_t ncap, const T* __restrict__ r,
                                               T* __restrict__ e, int sweeps) {
  constexpr int N = D * D * D;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * N;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g / N];
    int o = (int)(g % N);
    size_t i = (size_t)b * N + o;
    double dinv = (double)w[4 * ncap + i];
    double e1c = kOmega * dinv * (double)r[i];
    if (sweeps == 1 || dinv == 0) {
      e[i] = (T)e1c;
      continue;
    }
    int x = o % D, y = (o / D) % D, z = o / (D * D);
    double s = (double)w[3 * ncap + i] * e1c;
    for (int a = 0; a < 3; ++a) {
      double wl = (double)w[a * ncap + i];
      int p[3] = {x, y, z};
      p[a] -= 1;
      int64_t n = lidx<D>(nbr, b, p[0], p[1], p[2]);
      if (wl != 0 && n >= 0) s -= wl * kOmega * (double)w[4 * ncap + n] * (double)r[n];
      p[a] += 2;
      n = lidx<D>(nbr, b, p[0], p[1], p[2]);
      if (n >= 0) {
        double wr = (double)w[a * ncap + n];
        if (wr != 0) s -= wr * kOmega * (double)w[4 * ncap + n] * (double)r[n];
      }
    }
    e[i] = (T)(e1c + kOmega * dinv * ((double)r[i] - s));
  }
}

template <class T, int D>
__global__ void __launch_bounds__(256) k_restrict_l(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                    const T* __restrict__ w, size_t ncap, const T* __restrict__ r,
                                                    const T* __restrict__ e, T* __restrict__ rc, size_t ncapc) {
  constexpr int H = D / 2;
  constexpr int N = D * D * D;
  (void)ncapc;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * H * H * H;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g / (H * H * H)];
    int o = (int)(g % (H * H * H));
    int X = o % H, Y = (o / H) % H, Z = o / (H * H);
    double s = 0;
    for (int k = 0; k < 8; ++k) {
      int x = 2 * X + (k & 1), y = 2 * Y + ((k >> 1) & 1), z = 2 * Z + (k >> 2);
      size_t i = (size_t)b * N + x + D * y + D * D * z;
      if ((double)w[4 * ncap + i] == 0) continue;
      s += (double)r[i] - apply_l<T, D>(e, w, ncap, nbr, b, x, y, z, i, (double)e[i]);
    }
    rc[(size_t)b * H * H * H + o] = (T)s;
  }
}

// One Jacobi sweep at edge D, optionally adding the coarse correction (edge D/2) first.
template <class T, int D, bool WITH_COARSE>
__global__ void __launch_bounds__(256) k_jacobi_l(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                  const T* __restrict__ w, size_t ncap, const T* __restrict__ r,
                                                  const T* __restrict__ e, const T* __restrict__ ec, T* __restrict__ eout) {
  constexpr int N = D * D * D;
  constexpr int H = D / 2 > 0 ? D / 2 : 1;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * N;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g / N];
    int o = (int)(g % N);
    size_t i = (size_t)b * N + o;
    double dinv = (double)w[4 * ncap + i];
    if (dinv == 0) {
      eout[i] = (T)0;
      continue;
    }
    int x = o % D, y = (o / D) % D, z = o / (D * D);
    auto ev = [&](int64_t n) -> double {
      double v = (double)e[n];
      if (WITH_COARSE) {
        int nb = (int)(n / N);
        int no = (int)(n % N);
        int xx = no % D, yy = (no / D) % D, zz = no / (D * D);
        v += (double)ec[(size_t)nb * H * H * H + (xx >> 1) + H * (yy >> 1) + H * H * (zz >> 1)];
      }
      return v;
    };
    double ecc = ev((int64_t)i);
    double s = (double)w[3 * ncap + i] * ecc;
    for (int a = 0; a < 3; ++a) {
      double wl = (double)w[a * ncap + i];
      int p[3] = {x, y, z};
      p[a] -= 1;
      int64_t n = lidx<D>(nbr, b, p[0], p[1], p[2]);
      if (wl != 0 && n >= 0) s -= wl * ev(n);
      p[a] += 2;
      n = lidx<D>(nbr, b, p[0], p[1], p[2]);
      if (n >= 0) {
        double wr = (double)w[a * ncap + n];
        if (wr != 0) s -= wr * ev(n);
      }
    }
    eout[i] = (T)(ecc + kOmega * dinv * ((double)r[i] - s));
  }
}

// ------------------------------------------------------------ CG kernels
// Divergence (Policy_Divergence::Get_Divergence, src/Policy_Divergence.h:20-29)
// of speed buffer ib into r = -div (the residual of M x = -div at x = 0) and
// the partial sums of |div|^2.
__global__ void __launch_bounds__(256) k_divergence(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                    const uint16_t* __restrict__ fmask, const double* __restrict__ ux,
                                                    const double* __restrict__ uy, const double* __restrict__ uz,
                                                    double* __restrict__ rhs, double* __restrict__ x, int warm,
                                                    double* partial, Params P) {
  double bb = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    if (!(fmask[c] & kDomainBit)) {
      rhs[c] = 0.0;
      x[c] = 0.0;
      continue;
    }
    int x0 = o & 7, y0 = (o >> 3) & 7, z0 = o >> 6;
    const double* U[3] = {ux, uy, uz};
    double d = 0;
    for (int i = 0; i < 3; ++i) {
      d -= U[i][c] * P.ih[i];
      int p[3] = {x0, y0, z0};
      p[i] += 1;
      int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
      d += (n < 0 ? 0.0 : U[i][n]) * P.ih[i];
    }
    rhs[c] = -d;
    if (!warm) x[c] = 0.0;
    bb += d * d;
  }
  block_reduce2(bb, 0.0, partial);
}

// r = rhs - M x (used when starting from a non-zero x).
__global__ void __launch_bounds__(256) k_residual(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                  const uint16_t* __restrict__ fmask, const double* __restrict__ rhs,
                                                  const double* __restrict__ x, double* __restrict__ r, Params P) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    uint16_t m = fmask[c];
    if (!(m & kDomainBit)) {
      r[c] = 0.0;
      continue;
    }
    r[c] = rhs[c] - L0<double>::apply(x, nbr, b, o & 7, (o >> 3) & 7, o >> 6, m, x[c], P);
  }
}

__global__ void k_copy_vec(const int* __restrict__ blist, int nlive, const double* __restrict__ a, double* __restrict__ b) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = (int64_t)blist[g >> 9] * kCells + (g & 511);
    b[c] = a[c];
  }
}

// q = M p and partial p.q
__global__ void __launch_bounds__(256) k_spmv_dot(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                  const uint16_t* __restrict__ fmask, const double* __restrict__ p,
                                                  double* __restrict__ q, double* partial, Params P, const Scalars* ds) {
  if (ds->done) return;
  double pq = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    uint16_t m = fmask[c];
    if (!(m & kDomainBit)) {
      q[c] = 0.0;
      continue;
    }
    double pc = p[c];
    double v = L0<double>::apply(p, nbr, b, o & 7, (o >> 3) & 7, o >> 6, m, pc, P);
    q[c] = v;
    pq += pc * v;
  }
  block_reduce2(pq, 0.0, partial);
}

__global__ void k_fin_alpha(const double* partial, int nblk, Scalars* ds) {
  if (ds->done) return;
  double pq, unused;
  sum_partials(partial, nblk, &pq, &unused);
  if (threadIdx.x == 0) {
    ds->pq = pq;
    ds->alpha = pq != 0 ? ds->rz / pq : 0.0;
  }
}

// x += alpha p, r -= alpha q, partial r.r
__global__ void __launch_bounds__(256) k_axpy(const int* __restrict__ blist, int nlive, double* __restrict__ x,
                                              double* __restrict__ r, const double* __restrict__ p,
                                              const double* __restrict__ q, double* partial, const Scalars* ds) {
  if (ds->done) return;
  double a = ds->alpha;
  double rr = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = (int64_t)blist[g >> 9] * kCells + (g & 511);
    x[c] += a * p[c];
    double rv = r[c] - a * q[c];
    r[c] = rv;
    rr += rv * rv;
  }
  block_reduce2(rr, 0.0, partial);
}

__global__ void k_fin_rr(const double* partial, int nblk, Scalars* ds, double rtol2, int max_iters) {
  if (ds->done) return;
  double rr, unused;
  sum_partials(partial, nblk, &rr, &unused);
  if (threadIdx.x == 0) {
    ds->rr = rr;
    ds->iters += 1;
    if (rr <= rtol2 * ds->bnorm2 || ds->iters >= max_iters || !(rr == rr)) ds->done = 1;
  }
}

__global__ void k_fin_bnorm(const double* partial, int nblk, Scalars* ds) {
  double bb, unused;
  sum_partials(partial, nblk, &bb, &unused);
  if (threadIdx.x == 0) {
    ds->bnorm2 = bb;
    ds->rr = bb;
    ds->iters = 0;
    ds->done = bb == 0 ? 1 : 0;
  }
}

__global__ void k_fin_rr_initial(const double* partial, int nblk, Scalars* ds, double rtol2) {
  double rr, unused;
  sum_partials(partial, nblk, &rr, &unused);
  if (threadIdx.x == 0) {
    ds->rr = rr;
    if (rr <= rtol2 * ds->bnorm2) ds->done = 1;
  }
}

// r.r after a warm start residual
__global__ void __launch_bounds__(256) k_dot_rr(const int* __restrict__ blist, int nlive, const double* __restrict__ r,
                                                double* partial) {
  double rr = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = (int64_t)blist[g >> 9] * kCells + (g & 511);
    rr += r[c] * r[c];
  }
  block_reduce2(rr, 0.0, partial);
}

// beta = rz_new / rz (first call: p = z)
__global__ void k_fin_beta(const double* partial, int nblk, Scalars* ds, int first) {
  if (ds->done) return;
  double rz, unused;
  sum_partials(partial, nblk, &rz, &unused);
  if (threadIdx.x == 0) {
    ds->beta = first ? 0.0 : (ds->rz != 0 ? rz / ds->rz : 0.0);
    ds->rz = rz;
  }
}

__global__ void __launch_bounds__(256) k_update_p(const int* __restrict__ blist, int nlive, const double* __restrict__ z,
                                                  double* __restrict__ p, const Scalars* ds, int first) {
  if (ds->done) return;
  double be = ds->beta;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = (int64_t)blist[g >> 9] * kCells + (g & 511);
    p[c] = first ? z[c] : z[c] + be * p[c];
  }
}

// Pressure write-back and velocity correction, fused
// (src/Algorithms_Solve_Pressure.h:185-207): existing cells get p = x in the
// domain and 0 elsewhere; face i of a cell in the domain, or whose -e_i
// neighbour is, gets u_i -= p(c)/h_i - p(c-e_i)/h_i
// (Policy_Gradiant::Get_Gradiant, src/Policy_Gradiant.h:32-37) through the
// non-forced Set (const faces keep their value).
__global__ void __launch_bounds__(256) k_gradient(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                  const int8_t* __restrict__ lay, const uint8_t* __restrict__ type,
                                                  const uint8_t* __restrict__ flags, const double* __restrict__ x,
                                                  double* __restrict__ pres, double* ux, double* uy, double* uz,
                                                  Params P) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    if (lay[c] == kMissing) continue;
    bool dc = is_fluid(type[c]);
    double pc = dc ? x[c] : 0.0;
    pres[c] = pc;
    uint8_t fl = flags[c];
    int x0 = o & 7, y0 = (o >> 3) & 7, z0 = o >> 6;
    double* U[3] = {ux, uy, uz};
    for (int i = 0; i < 3; ++i) {
      int p[3] = {x0, y0, z0};
      p[i] -= 1;
      int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
      bool nexists = n >= 0 && lay[n] != kMissing;
      bool dn = nexists && is_fluid(type[n]);
      if (!(dc || dn)) continue;
      if (fl & (1u << i)) continue;
      double pn = nexists ? (dn ? x[n] : 0.0) : (n >= 0 ? pres[n] : 0.0);
      double gr = pc * P.ih[i];
      gr -= pn * P.ih[i];
      U[i][c] = U[i][c] - gr;
    }
  }
}

// max |div| over domain cells (the check of src/Algorithms_Solve_Pressure.h:208-219)
__global__ void __launch_bounds__(256) k_divmax(const int* __restrict__ blist, int nlive, const int* __restrict__ nbr,
                                                const uint16_t* __restrict__ fmask, const double* __restrict__ ux,
                                                const double* __restrict__ uy, const double* __restrict__ uz, Params P,
                                                Scalars* ds) {
  double mx = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int b = blist[g >> 9];
    int o = (int)(g & 511);
    int64_t c = (int64_t)b * kCells + o;
    if (!(fmask[c] & kDomainBit)) continue;
    int x0 = o & 7, y0 = (o >> 3) & 7, z0 = o >> 6;
    const double* U[3] = {ux, uy, uz};
    double d = 0;
    for (int i = 0; i < 3; ++i) {
      d -= U[i][c] * P.ih[i];
      int p[3] = {x0, y0, z0};
      p[i] += 1;
      int64_t n = lidx<8>(nbr, b, p[0], p[1], p[2]);
      d += (n < 0 ? 0.0 : U[i][n]) * P.ih[i];
    }
    d = fabs(d);
    if (d > mx) mx = d;
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&ds->div_bits, (unsigned long long)__double_as_longlong(mx));
}

__global__ void k_zero_div(Scalars* ds) { ds->div_bits = 0; }

// ------------------------------------------------------------ drivers
static int vec_grid(int nlive) {
  int64_t g = ((int64_t)nlive * kCells + 255) / 256;
  return (int)(g < kVecBlocks ? (g < 1 ? 1 : g) : kVecBlocks);
}

template <class T>
static void setup_weights(Ctx* c) {
  cudaStream_t st = c->stream;
  int n = c->nlive_host;
  size_t ncap[kLevels];
  for (int l = 0; l < kLevels; ++l) ncap[l] = (size_t)c->cap_bricks * (size_t)((8 >> l) * (8 >> l) * (8 >> l));
  T* w1 = (T*)c->mg_w[1];
  T* w2 = (T*)c->mg_w[2];
  T* w3 = (T*)c->mg_w[3];
  k_weights_l1<T><<<vec_grid(n), 256, 0, st>>>(c->blist, n, c->fmask, w1, ncap[1], c->dp); MAC_COUNT(c);
  k_weights_coarsen<T, 4><<<vec_grid(n), 256, 0, st>>>(c->blist, n, w1, ncap[1], w2, ncap[2]); MAC_COUNT(c);
  k_weights_coarsen<T, 2><<<vec_grid(n), 256, 0, st>>>(c->blist, n, w2, ncap[2], w3, ncap[3]); MAC_COUNT(c);
  k_weights_diag<T, 4><<<vec_grid(n), 256, 0, st>>>(c->blist, n, c->nbr, w1, ncap[1]); MAC_COUNT(c);
  k_weights_diag<T, 2><<<vec_grid(n), 256, 0, st>>>(c->blist, n, c->nbr, w2, ncap[2]); MAC_COUNT(c);
  k_weights_diag<T, 1><<<vec_grid(n), 256, 0, st>>>(c->blist, n, c->nbr, w3, ncap[3]); MAC_COUNT(c);
}

int setup_system(Ctx* c) {
  cudaStream_t st = c->stream;
  int n = c->nlive_host;
  prof_begin(c, PH_SETUP);
  k_zero_unknown<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
  if (n > 0) {
    k_fmask<<<vec_grid(n), 256, 0, st>>>(c->blist, n, c->nbr, c->lay, c->type, c->flags, c->fmask, c->ds); MAC_COUNT(c);
    if (c->mg_float) setup_weights<float>(c);
    else setup_weights<double>(c);
  }
  prof_end(c, PH_SETUP);
  c->system_ready = true;
  return check(cudaGetLastError());
}

template <class T>
static void vcycle(Ctx* c) {
  cudaStream_t st = c->stream;
  int n = c->nlive_host;
  size_t ncap[kLevels];
  for (int l = 0; l < kLevels; ++l) ncap[l] = (size_t)c->cap_bricks * (size_t)((8 >> l) * (8 >> l) * (8 >> l));
  T* e0 = (T*)c->mg_e[0];
  T* e0b = (T*)c->mg_e2[0];
  T* e1 = (T*)c->mg_e[1];
  T* e1b = (T*)c->mg_e2[1];
  T* e2 = (T*)c->mg_e[2];
  T* e2b = (T*)c->mg_e2[2];
  T* e3 = (T*)c->mg_e[3];
  T* e3b = (T*)c->mg_e2[3];
  T* r1 = (T*)c->mg_r[1];
  T* r2 = (T*)c->mg_r[2];
  T* r3 = (T*)c->mg_r[3];
  T* w1 = (T*)c->mg_w[1];
  T* w2 = (T*)c->mg_w[2];
  T* w3 = (T*)c->mg_w[3];
  int g0 = vec_grid(n);
  int g1 = grid_for((int64_t)n * 64, 256), g2 = grid_for((int64_t)n * 8, 256), g3 = grid_for(n, 256);
  // down
  k_pre0<T><<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, c->r, e0, c->dp); MAC_COUNT(c);
  k_restrict0<T><<<g1, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, c->r, e0, r1, c->dp); MAC_COUNT(c);
  k_pre_l<T, 4><<<g1, 256, 0, st>>>(c->blist, n, c->nbr, w1, ncap[1], r1, e1, 2); MAC_COUNT(c);
  k_restrict_l<T, 4><<<g2, 256, 0, st>>>(c->blist, n, c->nbr, w1, ncap[1], r1, e1, r2, ncap[2]); MAC_COUNT(c);
  k_pre_l<T, 2><<<g2, 256, 0, st>>>(c->blist, n, c->nbr, w2, ncap[2], r2, e2, 2); MAC_COUNT(c);
  k_restrict_l<T, 2><<<g3, 256, 0, st>>>(c->blist, n, c->nbr, w2, ncap[2], r2, e2, r3, ncap[3]); MAC_COUNT(c);
  // coarsest: Jacobi sweeps from zero
  k_pre_l<T, 1><<<g3, 256, 0, st>>>(c->blist, n, c->nbr, w3, ncap[3], r3, e3, 1); MAC_COUNT(c);
  for (int s = 1; s < kCoarseSweeps; ++s) {
    k_jacobi_l<T, 1, false><<<g3, 256, 0, st>>>(c->blist, n, c->nbr, w3, ncap[3], r3, e3, nullptr, e3b); MAC_COUNT(c);
    T* t = e3; e3 = e3b; e3b = t;
  }
  // up
  k_jacobi_l<T, 2, true><<<g2, 256, 0, st>>>(c->blist, n, c->nbr, w2, ncap[2], r2, e2, e3, e2b); MAC_COUNT(c);
  k_jacobi_l<T, 2, false><<<g2, 256, 0, st>>>(c->blist, n, c->nbr, w2, ncap[2], r2, e2b, nullptr, e2); MAC_COUNT(c);
  k_jacobi_l<T, 4, true><<<g1, 256, 0, st>>>(c->blist, n, c->nbr, w1, ncap[1], r1, e1, e2, e1b); MAC_COUNT(c);
  k_jacobi_l<T, 4, false><<<g1, 256, 0, st>>>(c->blist, n, c->nbr, w1, ncap[1], r1, e1b, nullptr, e1); MAC_COUNT(c);
  k_post0<T, true><<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, c->r, e0, e1, e0b, nullptr, nullptr, c->dp); MAC_COUNT(c);
  k_post0<T, false><<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, c->r, e0b, nullptr, nullptr, c->z, c->partial,
                                        c->dp); MAC_COUNT(c);
}

// Jacobi preconditioner (MAC_SOLVER_CG_FP64): z = r / diag, with the r.z partials.
__global__ void __launch_bounds__(256) k_jacobi_prec(const int* __restrict__ blist, int nlive,
                                                     const uint16_t* __restrict__ fmask, const double* __restrict__ r,
                                                     double* __restrict__ z, double* partial, Params P) {
  double rz = 0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < (int64_t)nlive * kCells;
       g += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = (int64_t)blist[g >> 9] * kCells + (g & 511);
    uint16_t m = fmask[c];
    double d = (m & kDomainBit) ? diag0(m, P) : 0.0;
    double v = d > 0 ? r[c] / d : 0.0;
    z[c] = v;
    rz += r[c] * v;
  }
  block_reduce2(rz, 0.0, partial);
}

static void precondition(Ctx* c) {
  if (c->prm.solver == MAC_SOLVER_CG_FP64) {
    int n = c->nlive_host;
    k_jacobi_prec<<<vec_grid(n), 256, 0, c->stream>>>(c->blist, n, c->fmask, c->r, c->z, c->partial, c->dp); MAC_COUNT(c);
  } else if (c->mg_float) {
    vcycle<float>(c);
  } else {
    vcycle<double>(c);
  }
}

int project(Ctx* c, int ib) {
  if (!c->system_ready) {
    int rc = setup_system(c);
    if (rc) return rc;
  }
  int n = c->nlive_host;
  if (n == 0) return MAC_OK;
  cudaStream_t st = c->stream;
  size_t cap = (size_t)c->cap_bricks * kCells;
  double* U[3] = {c->f64 + (size_t)(3 * ib) * cap, c->f64 + (size_t)(3 * ib + 1) * cap,
                  c->f64 + (size_t)(3 * ib + 2) * cap};
  int g0 = vec_grid(n);
  int warm = c->prm.warm_start ? 1 : 0;
  double rtol2 = c->prm.rtol * c->prm.rtol;
  // rhs (kept in b) and its norm
  prof_begin(c, PH_DIVERGENCE);
  k_divergence<<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, U[0], U[1], U[2], c->b, c->x, warm, c->partial,
                                   c->dp); MAC_COUNT(c);
  prof_end(c, PH_DIVERGENCE);
  k_fin_bnorm<<<1, 1024, 0, st>>>(c->partial, g0, c->ds); MAC_COUNT(c);
  if (warm) {
    k_residual<<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, c->b, c->x, c->r, c->dp); MAC_COUNT(c);
    k_dot_rr<<<g0, 256, 0, st>>>(c->blist, n, c->r, c->partial); MAC_COUNT(c);
    k_fin_rr_initial<<<1, 1024, 0, st>>>(c->partial, g0, c->ds, rtol2); MAC_COUNT(c);
  } else {
    k_copy_vec<<<g0, 256, 0, st>>>(c->blist, n, c->b, c->r); MAC_COUNT(c);
  }
  prof_begin(c, PH_VCYCLE);
  precondition(c);
  prof_end(c, PH_VCYCLE);
  k_fin_beta<<<1, 1024, 0, st>>>(c->partial, g0, c->ds, 1); MAC_COUNT(c);
  k_update_p<<<g0, 256, 0, st>>>(c->blist, n, c->z, c->pd, c->ds, 1); MAC_COUNT(c);
  int rc = check(cudaGetLastError());
  if (rc) return rc;
  int it = 0;
  int status = MAC_OK;
  while (true) {
    prof_begin(c, PH_SPMV);
    k_spmv_dot<<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, c->pd, c->q, c->partial, c->dp, c->ds); MAC_COUNT(c);
    prof_end(c, PH_SPMV);
    prof_begin(c, PH_CGVEC);
    k_fin_alpha<<<1, 1024, 0, st>>>(c->partial, g0, c->ds); MAC_COUNT(c);
    k_axpy<<<g0, 256, 0, st>>>(c->blist, n, c->x, c->r, c->pd, c->q, c->partial, c->ds); MAC_COUNT(c);
    k_fin_rr<<<1, 1024, 0, st>>>(c->partial, g0, c->ds, rtol2, c->prm.max_iters); MAC_COUNT(c);
    prof_end(c, PH_CGVEC);
    ++it;
    rc = read_scalars(c);
    if (rc) return rc;
    if (c->hs->done) break;
    prof_begin(c, PH_VCYCLE);
    precondition(c);
    prof_end(c, PH_VCYCLE);
    prof_begin(c, PH_CGVEC);
    k_fin_beta<<<1, 1024, 0, st>>>(c->partial, g0, c->ds, 0); MAC_COUNT(c);
    k_update_p<<<g0, 256, 0, st>>>(c->blist, n, c->z, c->pd, c->ds, 0); MAC_COUNT(c);
    prof_end(c, PH_CGVEC);
  }
  double relres = c->hs->bnorm2 > 0 ? sqrt(c->hs->rr / c->hs->bnorm2) : 0.0;
  c->stats.iterations = c->hs->iters;
  c->stats.total_iterations += c->hs->iters;
  c->stats.relres = relres;
  c->stats.solves += 1;
  c->stats.unknowns = c->hs->nunknown;
  if (!(relres <= c->prm.rtol)) status = MAC_ERR_NOT_CONVERGED;
  prof_begin(c, PH_GRADIENT);
  k_gradient<<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->lay, c->type, c->flags, c->x, c->f64 + (size_t)PRES * cap,
                                 U[0], U[1], U[2], c->dp); MAC_COUNT(c);
  prof_end(c, PH_GRADIENT);
  if (c->prm.div_check) {
    k_zero_div<<<1, 1, 0, st>>>(c->ds); MAC_COUNT(c);
    k_divmax<<<g0, 256, 0, st>>>(c->blist, n, c->nbr, c->fmask, U[0], U[1], U[2], c->dp, c->ds); MAC_COUNT(c);
    rc = read_scalars(c);
    if (rc) return rc;
    unsigned long long bits = c->hs->div_bits;
    std::memcpy(&c->stats.max_div, &bits, sizeof(double));
  }
  rc = check(cudaGetLastError());
  return rc ? rc : status;
}

}  // namespace mac
